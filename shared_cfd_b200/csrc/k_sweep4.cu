// k_sweep4.cu -- LU-SGS sweeps with a lane quad per cell, four cells per quad.
//
// Restates calc_next_step_implicit of store/time_scheme/LU-SGS/{2d,q2d}/time_lusgs_viscous.f90
// and NR/{2d,q2d}/time_NR_viscous.f90:30-108 with the split Jacobians of set_ABpm
// (sch_lusgs.raw.f90:1-141, NR/q2d/sch_NR.raw.f90:1-149) applied matrix-free:
//     (n1 A + n2 B) x = [Y;u;v;H] (n.m - un S) + un x + [0; n1 P; n2 P; un P],
//     P = dpdq . x,  S = sum of the species components,  A+- x = ((n1A+n2B)x +- nu x)/2.
// The cells are visited in the reference's dependency order (the forward sweep
// needs i-1 and j-1, the backward sweep i+1 and j+1); a schedule that honours
// those dependencies produces the reference's values whatever its timing.
//
// Schedule.
// * A warp owns a strip of R = 32 rows and at iteration t updates row r at
//   column t - r (the hyperplane wavefront, pipelined along the strip).
// * The Q = 4 lanes of a quad share one cell, each holding C = ceil(D/4) of its
//   D components: the last slot of quad lanes 0, 1, 2 holds rho u, rho v,
//   rho E, every other slot a species (L4::comp).  Quad g (g = 0..7) holds rows
//   g, g+8, g+16, g+24 ("sub-strips" k = 0..3), so every lane updates four
//   independent cells per iteration.  dpdq.x and the species sum of a cell are
//   formed with two xor shuffles inside its quad; x_u and x_v come from quad
//   lanes 0 and 1.
// * The j-1 neighbour's contribution (forward; j+1 backward) reaches row r
//   from row r-1 of the previous iteration by one shuffle over 4 lanes (quad 7
//   of sub-strip k-1 feeds quad 0 of sub-strip k); the i-1 (i+1) neighbour's
//   stays in registers.
// * Up to WPC strips of one plane form a task, run by one CTA with one warp per
//   strip.  A warp hands the contributions of its top row to the warp of the
//   next strip through a shared-memory ring of KCOL-column slots guarded by
//   full/empty mbarriers; the last warp of a task hands them to the next task
//   of the plane through global memory with a release/acquire progress counter,
//   in 8-column chunks.  Tasks are taken in ticket order, so a task only waits
//   for a task that is already running.
// * Inputs are repacked (k_pack4) into strip records
//     rec[strip][iteration][ scalars [SG][R][G] | lane fields [PG][R][Q][G] ]
//   (G elements = 16 bytes): the per-cell scalars once per row, the
//   per-component fields (x, dpdq, [Y,u,v,H], q_species) per lane, so that
//   shared-memory loads are conflict-free and one iteration of one strip is one
//   bulk copy, streamed PF - 1 iterations ahead into a per-warp ring.  Results
//   go back into the x fields of the same record; the backward sweep reads the
//   records with iterations and rows reversed; k_unpack4 applies q += omega*Dq.
// Every wait is bounded (kSpin4 polls); a wait that gives up sets SCFD_E_SPIN
// and the shared abort flag, and all warps leave.
#include "async_ptx.h"
#include "scfd_internal.h"

namespace scfd {

using namespace ptx;

namespace {

constexpr long long kSpin4 = 1ll << 22;
constexpr int KCOL = 2;    // columns per hand-off slot
constexpr int NSL = 16;    // hand-off slots per warp
constexpr int SB4 = 8;     // iterations per pack / unpack block
constexpr int PF_MAX = 8;  // deepest record ring of any instantiation
static_assert(8 % KCOL == 0, "hand-off slots must divide the 8-column chunk");

// Record blocks per warp ring (PF) and strips per task (WPC).  The records are
// larger than L2, so each bulk copy comes from HBM; a warp keeps PF - 1
// iterations in flight to cover that latency, and the rings of a task's warps
// must fit in shared memory (FP64 records are twice as large).
template <typename RT>
struct Cfg4 {
    static constexpr int PF = 8;
    static constexpr int WPC = sizeof(RT) == 4 ? 2 : 1;
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

__host__ __device__ constexpr int rup16(int b) { return (b + 15) & ~15; }

}  // namespace

template <typename RT, int NY>
struct L4 {
    static constexpr int Q = 4, K = 4, R8 = 8, R = K * R8;  // lanes per cell, sub-strips, rows
    static constexpr int D = NY + 3;
    static constexpr int C = (D + Q - 1) / Q;  // component slots per lane
    static constexpr int QC = Q * C;
    static constexpr int G = 16 / (int)sizeof(RT);
    static constexpr int NSC = 14;  // per-cell scalars
    static constexpr int SG = (NSC + G - 1) / G;
    static constexpr int PT = 4 * C;  // per-lane fields
    static constexpr int PG = (PT + G - 1) / G;
    static constexpr int XG = (C + G - 1) / G;  // groups holding x
    static constexpr int STEP = (SG * R + PG * R * Q) * G;
    // scalars: alpha, alpha*Area, 1/(1 - alpha*Area*dpdq_v), dpdq_v, then per
    // direction (A: i faces, B: j faces) ds/2, n1, n2, un, nu
    enum { AL = 0, AA, RQ, DPV, FA, N1A, N2A, UNA, NUA, FB, N1B, N2B, UNB, NUB };
    // per-lane fields, C slots each
    static constexpr int X = 0, DP = C, CV = 2 * C, QS = 3 * C;
    __host__ __device__ static constexpr int sc_off(int sc, int row) { return ((sc / G) * R + row) * G + sc % G; }
    __host__ __device__ static constexpr int pt_off(int f, int row, int c) {
        return SG * R * G + (((f / G) * R + row) * Q + c) * G + f % G;
    }
    __host__ __device__ static constexpr int sp_of(int c, int m) { return c < 3 ? c * (C - 1) + m : 3 * (C - 1) + m; }
    // component held in slot m of quad lane c (species 0..NY-1, then rho u,
    // rho v, rho E), or -1 for an unused slot
    __host__ __device__ static constexpr int comp(int c, int m) {
        return (m == C - 1 && c < 3) ? NY + c : (sp_of(c, m) < NY ? sp_of(c, m) : -1);
    }
};

// ---------------------------------------------------------------------------
// k_pack4: cell layout -> strip records.  One block packs SB4 iterations of one
// strip: thread (tx, r) forms the fields of cell (i = t0+tx-r+1, row r) into
// the shared-memory image of the record blocks (zero outside the plane), which
// is then stored contiguously.  Forms alpha, the spectral radii and dpdq of
// set_ABpm (sch_lusgs.raw.f90:27-50,134-136; NR/q2d/sch_NR.raw.f90:43-50,143-144).
// ---------------------------------------------------------------------------
template <typename RT, int NY>
__global__ void __launch_bounds__(SB4 * 32) k_pack4(View v, const int2* blk, const int4* strips, const long long* rec_off,
                                                    RT* rec, int nr_mode) {
    using L = L4<RT, NY>;
    using V = typename Vec16<RT>::type;
    constexpr int D = L::D, C = L::C, R = L::R, Q = L::Q, STEP = L::STEP;
    extern __shared__ __align__(128) unsigned char smraw[];
    RT* img = reinterpret_cast<RT*>(smraw);  // [SB4][STEP]
    const int2 b = blk[blockIdx.x];
    const int4 st = strips[b.x];
    const int p = st.x, s = st.y;
    const int ni = v.P.ni[p], nj = v.P.nj[p];
    const int nsteps = ni + R - 1;
    const int nt = min(SB4, nsteps - b.y);
    const int nthr = blockDim.x * blockDim.y, tid = threadIdx.y * blockDim.x + threadIdx.x;
    for (int e = tid; e < SB4 * STEP; e += nthr) img[e] = RT(0);
    __syncthreads();
    const int tx = threadIdx.x, g = threadIdx.y;
    const int cc = b.y + tx - g;
    const int j = R * s + 1 + g;
    if (tx < nt && cc >= 0 && cc < ni && j <= nj) {
        const long long N = v.ncell;
        const long long c = cidx(v.P, p, cc + 1, j);
        const double* w = v.w;
        const double rho = w[c], pr = w[3 * N + c];
        const double u = w[N + c], vv = w[2 * N + c];
        const double gamm = w[(D + 1) * N + c];
        const double g1 = gamm - 1.0;
        const double hvs = 0.5 * g1 * (u * u + vv * vv);
        const double cs = sqrt(gamm * pr / rho);
        const double n1a = v.vnci[c], n2a = v.vnci[N + c], n1b = v.vncj[c], n2b = v.vncj[N + c];
        const double una = n1a * u + n2a * vv, unb = n1b * u + n2b * vv;
        const double nuA = fabs(una) + cs, nuB = fabs(unb) + cs;
        const double dsa = v.dsci[c], dsb = v.dscj[c], vol = v.Vol[c];
        const double dtl = v.dt_mode == SCFD_DT_LOCAL ? v.dt_mat[c] : v.sc->dt_grbl;
        const double tmp = nr_mode ? 3.0 * vol / (2.0 * dtl) + dsa * nuA + dsb * nuB : vol / dtl + dsa * nuA + dsb * nuB;
        const double al = 1.0 / tmp;
        double aA = 0.0, rq = 1.0;
        if (v.dim == SCFD_DIM_Q2D) {
            aA = al * v.Area[c];
            rq = 1.0 / (1.0 - aA * (-g1 * vv));
        }
        RT* o = img + tx * STEP;
        const double scal[L::NSC] = {al, aA, rq, -g1 * vv, 0.5 * dsa, n1a, n2a, una, nuA, 0.5 * dsb, n1b, n2b, unb, nuB};
#pragma unroll
        for (int k = 0; k < L::NSC; ++k) o[L::sc_off(k, g)] = RT(scal[k]);
#pragma unroll
        for (int ql = 0; ql < Q; ++ql) {
#pragma unroll
            for (int m = 0; m < C; ++m) {
                const int k = L::comp(ql, m);
                if (k < 0) continue;
                double dp, cv, qs = 0.0;
                if (k < NY) {
                    dp = hvs + v.DHi[k * N + c];
                    cv = w[(4 + k) * N + c];
                    qs = v.q[k * N + c];
                } else if (k == NY) {
                    dp = -g1 * u;
                    cv = u;
                } else if (k == NY + 1) {
                    dp = 0.0;  // dpdq of rho v is the scalar DPV
                    cv = vv;
                } else {
                    dp = g1;
                    cv = w[(D + 2) * N + c];
                }
                o[L::pt_off(L::X + m, g, ql)] = RT(v.Dq[k * N + c]);
                o[L::pt_off(L::DP + m, g, ql)] = RT(dp);
                o[L::pt_off(L::CV + m, g, ql)] = RT(cv);
                o[L::pt_off(L::QS + m, g, ql)] = RT(qs);
            }
        }
    }
    __syncthreads();
    V* dst = reinterpret_cast<V*>(rec + rec_off[b.x] + (long long)b.y * STEP);
    const V* src = reinterpret_cast<const V*>(img);
    const int nv = nt * STEP / L::G;
    for (int e = tid; e < nv; e += nthr) dst[e] = src[e];
}

// ---------------------------------------------------------------------------
// the sweeps
// ---------------------------------------------------------------------------
struct Sweep4Args {
    const int4* tasks;          // (plane, first strip, strips, forward index of the first strip)
    int ntasks;
    const long long* rec_off;   // per forward strip: element offset of iteration 0
    void* rec;
    void* xfer;                 // per task: hand-off columns (QC values each)
    long long xstride;          // elements per task
    int* progress;              // per task: columns published
    int* ticket;
    double* partials;           // per forward strip: residual, omega limit
};

// Bounded wait on an mbarrier phase by every lane; the outcome is made uniform
// over the warp.  With `abortable` the wait also ends once another warp has
// given up.  Returns false if the wait gave up.
__device__ __forceinline__ bool warp_wait(unsigned long long* bar, unsigned parity, const View& v,
                                          bool abortable = true) {
    long long spins = 0;
    bool ok = true;
    while (!mbar_try_wait(bar, parity)) {
        if (++spins > kSpin4 ||
            (abortable && (spins & 4095) == 0 && *(volatile unsigned long long*)&v.sc->spin_abort)) {
            ok = false;
            break;
        }
    }
    return __all_sync(0xffffffffu, ok);
}

__device__ __forceinline__ void give_up(const View& v) {
    atomicExch(&v.sc->spin_abort, 1ull);
    atomicMax(&v.sc->status, SCFD_E_SPIN);
}

template <typename RT, int NY>
struct Smem4 {
    using L = L4<RT, NY>;
    static constexpr int PF4 = Cfg4<RT>::PF, WPC = Cfg4<RT>::WPC;
    static constexpr int RING = 0;
    static constexpr int HBUF = RING + WPC * PF4 * L::STEP * (int)sizeof(RT);
    static constexpr int XIN = HBUF + rup16(WPC * NSL * KCOL * L::QC * (int)sizeof(RT));
    static constexpr int BARS = XIN + rup16(8 * L::QC * (int)sizeof(RT));
    static constexpr int NBAR = WPC * (PF4 + 2 * NSL);
    static constexpr int TASK = BARS + NBAR * 8;
    static constexpr int BYTES = TASK + 16;
};

template <typename RT, int NY, int DIR>
__global__ void __launch_bounds__(32 * Cfg4<RT>::WPC) k_sweep4(View v, Sweep4Args a) {
    using L = L4<RT, NY>;
    using S = Smem4<RT, NY>;
    using V = typename Vec16<RT>::type;
    constexpr int PF4 = Cfg4<RT>::PF, WPC = Cfg4<RT>::WPC;
    constexpr int R = L::R, R8 = L::R8, K = L::K, Q = L::Q, C = L::C, QC = L::QC, G = L::G, STEP = L::STEP;
    constexpr int SG = L::SG, PG = L::PG, XG = L::XG;
    constexpr unsigned BLK = STEP * sizeof(RT);
    extern __shared__ __align__(128) unsigned char smraw[];
    RT* ring = reinterpret_cast<RT*>(smraw + S::RING);   // [WPC][PF4][STEP]
    RT* hbuf = reinterpret_cast<RT*>(smraw + S::HBUF);   // [WPC][NSL][KCOL][QC]
    RT* xin = reinterpret_cast<RT*>(smraw + S::XIN);     // [8][QC]
    unsigned long long* bars = reinterpret_cast<unsigned long long*>(smraw + S::BARS);
    int* s_task = reinterpret_cast<int*>(smraw + S::TASK);
    unsigned long long* fullb = bars + WPC * PF4;    // [WPC][NSL], producer = warp w
    unsigned long long* emptyb = fullb + WPC * NSL;  // [WPC][NSL]
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane / Q, c = lane % Q;  // quad (row within a sub-strip, sweep order), lane in the quad
    const bool nr = v.scheme == SCFD_SCHEME_NR;
    const bool q2d = v.dim == SCFD_DIM_Q2D;
    unsigned long long* tbar = bars + warp * PF4;
    if (threadIdx.x == 0) {
        for (int k = 0; k < S::NBAR; ++k) mbar_init(&bars[k], k < WPC * PF4 ? 1u : (unsigned)Q);
        mbar_init_fence();
    }
    __syncthreads();
    // record row of this lane's cell in sub-strip k: row r = 8k + g in sweep
    // order, row R-1-r of the record block in the backward sweep
    const int rf0 = DIR == 0 ? g : R - 1 - g;
    constexpr int RSTEP = DIR == 0 ? R8 : -R8;  // record-row step between sub-strips
    unsigned tphase = 0;              // parity of the next completion of each ring slot
    unsigned pend = 0;                // ring slots with a copy in flight
    long long hb_out = 0, hb_in = 0;  // hand-off slots filled / drained so far (all tasks)
    bool bail = false;
    for (;;) {
        if (threadIdx.x == 0) {
            int t = atomicAdd(a.ticket, 1);
            if (*(volatile unsigned long long*)&v.sc->spin_abort) t = a.ntasks;
            *s_task = t;
        }
        __syncthreads();
        const int tid = *s_task;
        __syncthreads();
        if (tid >= a.ntasks) break;
        const int4 tk = a.tasks[tid];
        const int p = tk.x, g0 = tk.y, nw = tk.z, fs0 = tk.w;
        if (warp >= nw || bail) continue;
        const int ni = v.P.ni[p], nj = v.P.nj[p];
        const int nstr = (nj + R - 1) / R;
        const int s = DIR == 0 ? g0 + warp : g0 + nw - 1 - warp;
        const int fs = fs0 + (s - g0);
        const int nsteps = ni + R - 1;
        const int nblk8 = (nsteps + 7) / 8;
        const int in_kind = warp > 0 ? 2 : ((DIR == 0 ? g0 > 0 : g0 + nw < nstr) ? 1 : 0);
        const int out_kind = warp < nw - 1 ? 2 : ((DIR == 0 ? g0 + nw < nstr : g0 > 0) ? 1 : 0);
        RT* srec = reinterpret_cast<RT*>(a.rec) + a.rec_off[fs];
        const RT* rd = srec + (DIR == 0 ? 0 : (long long)(nsteps - 1) * STEP);
        const long long gstep = DIR == 0 ? STEP : -STEP;
        RT* ring_w = ring + warp * PF4 * STEP;
        RT* hout = hbuf + warp * NSL * KCOL * QC;
        const RT* hin = hbuf + (warp > 0 ? warp - 1 : 0) * NSL * KCOL * QC;
        unsigned long long* full_in = fullb + (warp > 0 ? warp - 1 : 0) * NSL;
        unsigned long long* empty_in = emptyb + (warp > 0 ? warp - 1 : 0) * NSL;
        unsigned long long* full_out = fullb + warp * NSL;
        unsigned long long* empty_out = emptyb + warp * NSL;
        RT* xout = reinterpret_cast<RT*>(a.xfer) + (long long)tid * a.xstride;
        const RT* xsrc = reinterpret_cast<const RT*>(a.xfer) + (long long)(tid > 0 ? tid - 1 : 0) * a.xstride;
        if (lane == 0) {
#pragma unroll
            for (int tt = 0; tt < PF4 - 1; ++tt) {
                mbar_expect_tx(&tbar[tt], BLK);
                tma_bulk_g2s(ring_w + tt * STEP, rd + tt * gstep, BLK, &tbar[tt]);
            }
        }
        pend |= (1u << (PF4 - 1)) - 1u;
        RT outA[K][C], outB[K][C];
#pragma unroll
        for (int k = 0; k < K; ++k)
#pragma unroll
            for (int m = 0; m < C; ++m) {
                outA[k][m] = RT(0);
                outB[k][m] = RT(0);
            }
        double res = 0.0;
        double on = __longlong_as_double(0x7FF0000000000000ll), od = 1.0;  // omega candidate q / (-Dq)
        RT* gblk = const_cast<RT*>(rd) + L::pt_off(0, rf0, c);
        for (int tb = 0; tb < nblk8 && !bail; ++tb) {
            const int t0 = tb * 8;
            if (in_kind == 1 && t0 < ni) {
                const int need = t0 + 8 < ni ? t0 + 8 : ni;
                bool ok = true;
                if (lane == 0) {
                    long long spins = 0;
                    while (ld_acquire_gpu(a.progress + tid - 1) < need) {
                        if (++spins > kSpin4 || *(volatile unsigned long long*)&v.sc->spin_abort) {
                            ok = false;
                            break;
                        }
                    }
                }
                if (!__shfl_sync(0xffffffffu, ok, 0)) {
                    if (lane == 0) give_up(v);
                    bail = true;
                    break;
                }
                __syncwarp();
                for (int e = lane; e < 8 * QC; e += 32) xin[e] = __ldcg(xsrc + (long long)t0 * QC + e);
                __syncwarp();
            }
#pragma unroll 1
            for (int h = 0; h < 8 && !bail; h += KCOL) {
#pragma unroll
                for (int uu = 0; uu < KCOL; ++uu) {
                    const int u = h + uu;
                    const int t = t0 + u;
                    {
                        const int sl2 = (t + PF4 - 1) % PF4;
                        if (lane == 0) {
                            mbar_expect_tx(&tbar[sl2], BLK);
                            tma_bulk_g2s(ring_w + sl2 * STEP, rd + (long long)(t + PF4 - 1) * gstep, BLK, &tbar[sl2]);
                        }
                        pend |= 1u << sl2;
                    }
                    // contribution of the strip below (forward) / above (backward) to row 0
                    RT hv[C];
#pragma unroll
                    for (int m = 0; m < C; ++m) hv[m] = RT(0);
                    if (in_kind == 2) {
                        if (t < ni) {
                            const long long n = hb_in + (t0 + h) / KCOL;
                            const int sl = (int)(n % NSL);
                            if (uu == 0 && !warp_wait(&full_in[sl], (unsigned)((n / NSL) & 1), v)) {
                                if (lane == 0) give_up(v);
                                bail = true;
                                break;
                            }
                            if (g == 0) {
                                const RT* hp = hin + (sl * KCOL + uu) * QC + c * C;
#pragma unroll
                                for (int m = 0; m < C; ++m) hv[m] = hp[m];
                                if (uu == KCOL - 1 || t == ni - 1) mbar_arrive(&empty_in[sl]);
                            }
                        }
                    } else if (in_kind == 1) {
                        if (t < ni && g == 0) {
#pragma unroll
                            for (int m = 0; m < C; ++m) hv[m] = xin[u * QC + c * C + m];
                        }
                    }
                    // row r gets row r-1's contribution of the previous iteration: quad
                    // g-1 of the same sub-strip, or quad 7 of sub-strip k-1 for g = 0
                    RT inB[K][C];
#pragma unroll
                    for (int k = 0; k < K; ++k)
#pragma unroll
                        for (int m = 0; m < C; ++m) {
                            const RT snd = (k > 0 && g == R8 - 1) ? outB[k - 1][m] : outB[k][m];
                            const RT rcv = __shfl_sync(0xffffffffu, snd, (lane + 32 - Q) & 31);
                            inB[k][m] = (k == 0 && g == 0) ? hv[m] : rcv;
                        }
                    const int slot = t % PF4;
                    if (!warp_wait(&tbar[slot], (tphase >> slot) & 1u, v)) {
                        if (lane == 0) give_up(v);
                        bail = true;
                        break;
                    }
                    tphase ^= 1u << slot;
                    pend &= ~(1u << slot);
                    const RT* blk = ring_w + slot * STEP;
#pragma unroll
                    for (int k = 0; k < K; ++k) {
                        const int rf = rf0 + k * RSTEP;
                        RT sc[SG * G];
#pragma unroll
                        for (int e = 0; e < SG; ++e)
                            *reinterpret_cast<V*>(&sc[e * G]) = *reinterpret_cast<const V*>(blk + (e * R + rf) * G);
                        RT f[PG * G];
#pragma unroll
                        for (int e = 0; e < PG; ++e)
                            *reinterpret_cast<V*>(&f[e * G]) =
                                *reinterpret_cast<const V*>(blk + SG * R * G + ((e * R + rf) * Q + c) * G);
                        const RT al = sc[L::AL];
                        RT x[C];
#pragma unroll
                        for (int m = 0; m < C; ++m)
                            x[m] = DIR == 0 ? al * (f[L::X + m] + (outA[k][m] + inB[k][m]))
                                            : f[L::X + m] - al * (outA[k][m] + inB[k][m]);
                        // quad sums: dpdq.x without the rho v term, and the species sum
                        RT Pw = RT(0), Sp = RT(0);
#pragma unroll
                        for (int m = 0; m < C; ++m) Pw += f[L::DP + m] * x[m];
#pragma unroll
                        for (int m = 0; m < C - 1; ++m) Sp += x[m];
                        if (c == 3) Sp += x[C - 1];
                        Pw += __shfl_xor_sync(0xffffffffu, Pw, 1);
                        Sp += __shfl_xor_sync(0xffffffffu, Sp, 1);
                        Pw += __shfl_xor_sync(0xffffffffu, Pw, 2);
                        Sp += __shfl_xor_sync(0xffffffffu, Sp, 2);
                        const RT xu = __shfl_sync(0xffffffffu, x[C - 1], lane & ~3);
                        RT xv = __shfl_sync(0xffffffffu, x[C - 1], (lane & ~3) | 1);
                        // forward q2d: semi-implicit pressure source (q2d time_lusgs_viscous.f90:38-44)
                        if (DIR == 0 && q2d) {
                            xv = (xv + sc[L::AA] * Pw) * sc[L::RQ];
                            if (c == 1) x[C - 1] = xv;
                        }
                        const RT P = Pw + sc[L::DPV] * xv;
#pragma unroll
                        for (int dn = 0; dn < 2; ++dn) {
                            const int b0 = dn == 0 ? L::FA : L::FB;
                            const RT fa = sc[b0], n1 = sc[b0 + 1], n2 = sc[b0 + 2], un = sc[b0 + 3], nu = sc[b0 + 4];
                            const RT base_ = n1 * xu + n2 * xv - un * Sp;
                            const RT lam = DIR == 0 ? un + nu : un - nu;
                            const RT pc = c == 0 ? n1 : (c == 1 ? n2 : (c == 2 ? un : RT(0)));
                            RT* o = dn == 0 ? outA[k] : outB[k];
#pragma unroll
                            for (int m = 0; m < C - 1; ++m) o[m] = fa * (f[L::CV + m] * base_ + lam * x[m]);
                            o[C - 1] = fa * (f[L::CV + C - 1] * base_ + lam * x[C - 1] + pc * P);
                        }
                        // result back into the record block (16-byte stores)
#pragma unroll
                        for (int m = 0; m < C; ++m) f[L::X + m] = x[m];
#pragma unroll
                        for (int e = 0; e < XG; ++e)
                            *reinterpret_cast<V*>(gblk + (k * RSTEP + e * R) * Q * G) = *reinterpret_cast<V*>(&f[e * G]);
                        if (DIR == 1 && nr) {
                            if (c == 2) {
                                const double dE = double(x[C - 1]);
                                res = res + dE * dE;
                            }
#pragma unroll
                            for (int m = 0; m < C; ++m) {
                                if (m < C - 1 || c == 3) {
                                    // smallest q_k/(-Dq_k) over Dq_k < 0, compared by cross-multiplication
                                    const double dk = double(x[m]);
                                    const double qn = double(f[L::QS + m]), qd = -dk;
                                    if (dk < 0.0 && qn * od < on * qd) {
                                        on = qn;
                                        od = qd;
                                    }
                                }
                            }
                        }
                    }
                    gblk += gstep;
                    // hand the top row's contribution (quad 7 of sub-strip K-1) to the next strip
                    const int cc = t - (R - 1);
                    if (out_kind == 2) {
                        if (cc >= 0 && cc < ni) {
                            const int ck = ((uu - (R - 1)) % KCOL + KCOL) % KCOL;  // == cc % KCOL
                            const long long n = hb_out + cc / KCOL;
                            const int sl = (int)(n % NSL);
                            if (ck == 0 && n >= NSL &&
                                !warp_wait(&empty_out[sl], (unsigned)(((n / NSL) - 1) & 1), v)) {
                                if (lane == 0) give_up(v);
                                bail = true;
                                break;
                            }
                            if (g == R8 - 1) {
                                RT* hp = hout + (sl * KCOL + ck) * QC + c * C;
#pragma unroll
                                for (int m = 0; m < C; ++m) hp[m] = outB[K - 1][m];
                                if (ck == KCOL - 1 || cc == ni - 1) mbar_arrive(&full_out[sl]);
                            }
                        }
                    } else if (out_kind == 1) {
                        if (cc >= 0 && cc < ni && g == R8 - 1) {
#pragma unroll
                            for (int m = 0; m < C; ++m) xout[(long long)cc * QC + c * C + m] = outB[K - 1][m];
                        }
                    }
                    __syncwarp();
                }
            }
            if (bail) break;
            if (out_kind == 1) {
                const int done = t0 + 8 - (R - 1) < ni ? t0 + 8 - (R - 1) : ni;
                if (done > 0) {
                    if (g == R8 - 1) __threadfence();
                    __syncwarp();
                    if (lane == (R8 - 1) * Q) st_release_gpu(a.progress + tid, done);
                }
            }
        }
        // let the copies still in flight (prefetches past the end, or all of them
        // after a wait gave up) land before the ring is reused or the CTA exits
#pragma unroll
        for (int k = 0; k < PF4; ++k) {
            if (!((pend >> k) & 1u)) continue;
            if (!warp_wait(&tbar[k], (tphase >> k) & 1u, v, false)) {
                if (lane == 0) give_up(v);
                bail = true;
                break;
            }
            tphase ^= 1u << k;
            pend &= ~(1u << k);
        }
        if (bail) continue;
        if (in_kind == 2) hb_in += (ni + KCOL - 1) / KCOL;
        if (out_kind == 2) hb_out += (ni + KCOL - 1) / KCOL;
        if (DIR == 1 && nr) {
            for (int o = 16; o > 0; o >>= 1) {
                res += __shfl_xor_sync(0xffffffffu, res, o);
                const double on2 = __shfl_xor_sync(0xffffffffu, on, o), od2 = __shfl_xor_sync(0xffffffffu, od, o);
                if (on2 * od < on * od2) {
                    on = on2;
                    od = od2;
                }
            }
            if (lane == 0) {
                const double om = on / od * v.dq_max;  // -q/Dq*Dqmax of the limiting cell
                a.partials[2 * fs] = res;
                a.partials[2 * fs + 1] = om;
                if (om < v.omega_min) atomicMax(&v.sc->status, SCFD_E_OMEGA);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// k_unpack4: q += omega * Dq from the records (LU-SGS: omega = 1; NR: the
// positivity-limited omega reduced from the per-strip partials,
// time_NR_viscous.f90:86-108).  One block per SB4 iterations of one strip; the
// x fields are staged in shared memory and written back along i.
// ---------------------------------------------------------------------------
template <typename RT, int NY>
__global__ void __launch_bounds__(SB4 * 32) k_unpack4(View v, const int2* blk, const int4* strips,
                                                      const long long* rec_off, const RT* rec, const double* partials,
                                                      int nstrips, int nr_mode, int inner) {
    using L = L4<RT, NY>;
    constexpr int R = L::R, Q = L::Q, C = L::C, G = L::G, STEP = L::STEP, XG = L::XG;
    constexpr int XR = XG * R * Q * G;  // x part of one record block
    constexpr int NT = SB4 * 32;
    __shared__ RT tile[SB4][XR];
    __shared__ double s_res[NT], s_om[NT];
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    double om = 1.0;
    if (nr_mode) {
        double r = 0.0, o = 1e300;
        for (int k = tid; k < nstrips; k += NT) {
            r += partials[2 * k];
            o = fmin(o, partials[2 * k + 1]);
        }
        s_res[tid] = r;
        s_om[tid] = o;
        __syncthreads();
        for (int h = NT / 2; h > 0; h >>= 1) {
            if (tid < h) {
                s_res[tid] += s_res[tid + h];
                s_om[tid] = fmin(s_om[tid], s_om[tid + h]);
            }
            __syncthreads();
        }
        om = fmin(v.omega_max, s_om[0]);
        if (blockIdx.x == 0 && tid == 0) {
            if (inner == 1) v.sc->res1 = s_res[0];
            v.sc->res = s_res[0];
            v.sc->omega = om;
        }
        if (v.sc->status == SCFD_E_OMEGA) return;
    }
    const int2 b = blk[blockIdx.x];
    const int4 st = strips[b.x];
    const int p = st.x, s = st.y;
    const int ni = v.P.ni[p], nj = v.P.nj[p];
    const int nt = min(SB4, ni + R - 1 - b.y);
    const RT* in = rec + rec_off[b.x] + (long long)b.y * STEP + L::SG * R * G;
    for (int e = tid; e < SB4 * XR; e += NT) {
        const int tt = e / XR, k = e % XR;
        tile[tt][k] = tt < nt ? in[(long long)tt * STEP + k] : RT(0);
    }
    __syncthreads();
    const int tx = threadIdx.x, g = threadIdx.y;
    const int cc = b.y + tx - g, j = R * s + 1 + g;
    if (tx >= nt || cc < 0 || cc >= ni || j > nj) return;
    const long long N = v.ncell;
    const long long c = cidx(v.P, p, cc + 1, j);
#pragma unroll
    for (int ql = 0; ql < Q; ++ql) {
#pragma unroll
        for (int m = 0; m < C; ++m) {
            const int k = L::comp(ql, m);
            if (k < 0) continue;
            const double d = double(tile[tx][((m / G) * R + g) * Q * G + ql * G + m % G]);
            v.q[k * N + c] = nr_mode ? v.q[k * N + c] + om * d : v.q[k * N + c] + d;
        }
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
int sweep4_rows() { return L4<float, 1>::R; }
int sweep4_strips_per_task(bool mixed) { return mixed ? Cfg4<float>::WPC : Cfg4<double>::WPC; }
int sweep4_pad_steps() { return 8 + PF_MAX; }
int sweep4_steps_per_block() { return SB4; }

size_t sweep4_record_elems(int ny, bool mixed, int* qc) {
    switch (ny) {
        case 1: *qc = L4<float, 1>::QC; return mixed ? L4<float, 1>::STEP : L4<double, 1>::STEP;
        case 8: *qc = L4<float, 8>::QC; return mixed ? L4<float, 8>::STEP : L4<double, 8>::STEP;
        case 9: *qc = L4<float, 9>::QC; return mixed ? L4<float, 9>::STEP : L4<double, 9>::STEP;
        default: *qc = 0; return 0;
    }
}

template <typename RT, int NY, int DIR>
static void sweep4_launch(const View& v, cudaStream_t s, const Sweep4& w) {
    using Sm = Smem4<RT, NY>;
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_sweep4<RT, NY, DIR>, cudaFuncAttributeMaxDynamicSharedMemorySize, Sm::BYTES);
        attr = true;
    }
    Sweep4Args a{DIR == 0 ? w.tasks_f : w.tasks_b, w.ntasks, w.rec_off, w.rec, w.xfer, w.xstride,
                 w.progress + (DIR == 0 ? 0 : w.ntasks), w.tickets + (DIR == 0 ? 0 : 1), w.partials};
    k_sweep4<RT, NY, DIR><<<w.ntasks, 32 * Cfg4<RT>::WPC, Sm::BYTES, s>>>(v, a);
}

template <typename RT, int NY>
static void run4(const View& v, cudaStream_t s, const Sweep4& w, int what, int inner) {
    const bool nr = v.scheme == SCFD_SCHEME_NR;
    if (what == 0) {
        const size_t smem = (size_t)SB4 * L4<RT, NY>::STEP * sizeof(RT);
        static bool attr = false;
        if (!attr) {
            cudaFuncSetAttribute(k_pack4<RT, NY>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            attr = true;
        }
        k_pack4<RT, NY><<<w.nblk, dim3(SB4, L4<RT, NY>::R), smem, s>>>(v, w.blk, w.strips, w.rec_off,
                                                                      reinterpret_cast<RT*>(w.rec), nr ? 1 : 0);
    } else if (what == 3) {
        k_unpack4<RT, NY><<<w.nblk, dim3(SB4, L4<RT, NY>::R), 0, s>>>(v, w.blk, w.strips, w.rec_off,
                                                                     reinterpret_cast<const RT*>(w.rec), w.partials,
                                                                     w.nstrips, nr ? 1 : 0, inner);
    } else if (what == 1) {
        sweep4_launch<RT, NY, 0>(v, s, w);
    } else {
        sweep4_launch<RT, NY, 1>(v, s, w);
    }
}

// what: 0 pack, 1 forward sweep, 2 backward sweep, 3 unpack/update
int launch_sweep4(const View& v, cudaStream_t s, const Sweep4& w, int what, int inner) {
    const bool mixed = v.precision == SCFD_PREC_MIXED;
    switch (v.nY) {
        case 1: if (mixed) run4<float, 1>(v, s, w, what, inner); else run4<double, 1>(v, s, w, what, inner); return 1;
        case 8: if (mixed) run4<float, 8>(v, s, w, what, inner); else run4<double, 8>(v, s, w, what, inner); return 1;
        case 9: if (mixed) run4<float, 9>(v, s, w, what, inner); else run4<double, 9>(v, s, w, what, inner); return 1;
        default: return 0;
    }
}

}  // namespace scfd
