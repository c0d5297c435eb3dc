// k_wave.cu -- LU-SGS sweeps as cluster wavefronts.
//
// Restates calc_next_step_implicit of store/time_scheme/LU-SGS/{2d,q2d}/time_lusgs_viscous.f90
// and NR/{2d,q2d}/time_NR_viscous.f90:30-108 with the split Jacobians of set_ABpm
// (sch_lusgs.raw.f90:1-141, NR/q2d/sch_NR.raw.f90:1-149), applied matrix-free.
//
// Schedule.  A strip is 32 rows of one plane; lane l of a strip's compute warp
// owns row 32 s + 1 + l and at sweep step t updates column t - l (the
// hyperplane order i + j of the reference, lane l lagging lane l - 1 by one
// step).  The i - 1 neighbour's product is in the lane's registers, the j - 1
// neighbour's arrives from lane l - 1 by __shfl_up, and the bottom row of a
// strip takes the top row of the strip below (lane 31 of that warp) through a
// hand-off ring in shared memory.
//
// A task is up to 8 consecutive strips of one plane, run by one thread-block
// cluster of 8 CTAs (CTA rank r on the task's strip r).  Strip r's lane 31
// stages its row in its own shared memory; every HK columns it moves the chunk
// with one bulk copy into CTA r + 1's hand-off ring (distributed shared
// memory), completing a transaction count on an mbarrier of the receiving
// CTA; the receiver releases each chunk with a remote arrive.  A task with a successor
// holds 8 strips, so only rank 7 ever publishes to global memory and ranks
// 0-6 only to the next CTA.  Between tasks of one plane the
// top row travels through global memory: the last CTA's helper warp copies it
// out and publishes a progress counter (release), the next task's rank-0
// helper polls it (acquire) and bulk-copies the chunk into its own ring.
// Tasks are taken from a ticket counter in dependency order, so a cluster only
// ever waits for tasks that are already running.
//
// Each CTA has one compute warp and one helper warp.  The compute warp does
// the wavefront only: no global loads, stores or fences in its step loop.  The
// helper streams the strip's records through a ring of slots (bulk copies
// completing on mbarriers), writes the results back with bulk stores, and moves
// the hand-off chunks on (to the next CTA, or through global memory).  Every wait is bounded; a wait that gives up sets
// SCFD_E_SPIN and the kernel winds down instead of hanging.
//
// Records (k_pack, in the cell order of the sweep):
//   X[strip][step t][gx][lane l][G]  x(1:D): right-hand side, forward result, Dq
//   C[strip][step t][gc][lane l][G]  the cell's coefficients (CF below)
// for the cell (i = t - l + 1, j = 32 s + 1 + l), G = 16 bytes of values, so a
// lane reads its cell with 16-byte shared-memory loads.  The backward sweep
// walks the same records with steps and lanes reversed.  k_unpack applies
// q += omega Dq back in the cell layout.
#include "async_ptx.h"
#include "scfd_internal.h"

namespace scfd {

using namespace ptx;

namespace {

constexpr int CL = 8;    // CTAs per cluster = strips per task
constexpr int HK = 4;    // hand-off columns per chunk
constexpr int HS = 32;   // hand-off ring chunks
constexpr int kPadSteps = 8;  // zero step blocks before and after each strip's records
constexpr long long kSpin = 1ll << 22;

// hand-off chunks of a strip's top row for a plane of ni columns: chunk j
// holds the columns 4j-3 .. 4j (HK = 4), j = 0 .. (ni + 2) / 4
__host__ __device__ constexpr int chunks_of(int ni) { return (ni + 2) / 4 + 1; }

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

}  // namespace

// Coefficient fields of one cell (set_ABpm's quantities, sch_lusgs.raw.f90:27-50,134-136;
// NR/q2d/sch_NR.raw.f90:43-50,143-144), formed in FP64 by k_pack:
//   AL            alpha = 1/(Vol/dt + dsci nuA + dscj nuB)   (NR: 3 Vol/(2 dt))
//   AA, RQ        alpha*Area and 1/(1 - alpha*Area*dpdq_my)  (q2d pressure source)
//   G1            gamma - 1
//   DP(1:nY)      dpdq of the species: 0.5 g1 |u|^2 + DHi
//   Y(1:nY), U, V, H    the primitive vector (Y, u, v, H) of the split Jacobians
//   per direction d (A: i, ds = dsci, n = vnci; B: j, ds = dscj, n = vncj), with
//   fa = ds/2, un = n.u and nu = |un| + sound speed:
//   P1 = fa n1, P2 = fa n2, PU = fa un, LP = fa (un + nu), LM = fa (un - nu)
template <int NY>
struct CF {
    static constexpr int AL = 0, AA = 1, RQ = 2, G1 = 3, DP = 4, Y = DP + NY, U = Y + NY, V = U + 1, H = U + 2,
                         PA = U + 3, PB = PA + 5, NC = PB + 5;
    // offsets within a direction's block
    static constexpr int P1 = 0, P2 = 1, PU = 2, LP = 3, LM = 4;
};
template <typename RT, int NY>
struct WL {
    static constexpr int G = 16 / (int)sizeof(RT);
    static constexpr int D = NY + 3;
    static constexpr int NGX = (D + G - 1) / G;
    static constexpr int NGC = (CF<NY>::NC + G - 1) / G;
    static constexpr int XS = NGX * 32 * G;  // elements of one step block of X
    static constexpr int CS = NGC * 32 * G;  // and of C
    static constexpr int D4 = NGX * G;       // hand-off column (D values, padded)
    // steps per record slot (one bulk copy, one wait and one release per slot) and
    // slots in the ring.  FP32: 4 slots of 8 steps (fewer waits per step; 0.641 ->
    // 0.61 ms per sweep pair at 786 k cells).  FP64: the same shared memory holds
    // 16 steps, and 2 slots of 8 leave too short a prefetch (0.893 -> 0.950 ms),
    // so 4 slots of 4.
    static constexpr int SPB = sizeof(RT) == 4 ? 8 : 4;
    static constexpr int PFB = 4;
    static constexpr size_t SMEM = sizeof(RT) * ((size_t)PFB * SPB * (XS + CS) + 2 * HS * HK * D4) +
                                   8 * (2 * PFB + 5 * HS) + 16;
};

// ---------------------------------------------------------------------------
// k_pack: cell layout -> records (32 steps x 32 lanes of one strip per block;
// reads coalesced along i, writes coalesced 16-byte groups through a
// shared-memory transpose).
// ---------------------------------------------------------------------------
template <typename T, int NY>
__global__ void __launch_bounds__(1024) k_pack(View v, const int2* blk, const int4* strips, const long long* step_off,
                                               T* X, T* Cr, int nr_mode) {
    using F = CF<NY>;
    using L = WL<T, NY>;
    constexpr int D = NY + 3, G = L::G, NGX = L::NGX, NGC = L::NGC, NG = NGX + NGC;
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
    double al = 0.0, u = 0.0, vv = 0.0, g1 = 0.0, hvs = 0.0, aA = 0.0, rq = 1.0, cs = 0.0;
    double dir[2][5] = {};  // P1, P2, PU, LP, LM of directions A (i) and B (j)
    if (ok) {
        const double* w = v.w;
        const double rho = w[c];
        const double pr = w[3 * N + c];
        u = w[N + c];
        vv = w[2 * N + c];
        const double gamm = w[(D + 1) * N + c];
        g1 = gamm - 1.0;
        hvs = 0.5 * g1 * (u * u + vv * vv);
        cs = sqrt(gamm * pr / rho);
        const double nuA = fabs(v.vnci[c] * u + v.vnci[N + c] * vv) + cs;
        const double nuB = fabs(v.vncj[c] * u + v.vncj[N + c] * vv) + cs;
        const double dsa = v.dsci[c], dsb = v.dscj[c], vol = v.Vol[c];
        for (int d = 0; d < 2; ++d) {
            const double fa = 0.5 * (d == 0 ? dsa : dsb);
            const double n1 = d == 0 ? v.vnci[c] : v.vncj[c], n2 = d == 0 ? v.vnci[N + c] : v.vncj[N + c];
            const double un = n1 * u + n2 * vv, nu = fabs(un) + cs;
            dir[d][0] = fa * n1;
            dir[d][1] = fa * n2;
            dir[d][2] = fa * un;
            dir[d][3] = fa * (un + nu);
            dir[d][4] = fa * (un - nu);
        }
        const double dtl = v.dt_mode == SCFD_DT_LOCAL ? v.dt_mat[c] : v.sc->dt_grbl;
        const double tmp = nr_mode ? 3.0 * vol / (2.0 * dtl) + dsa * nuA + dsb * nuB : vol / dtl + dsa * nuA + dsb * nuB;
        al = 1.0 / tmp;
        if (v.dim == SCFD_DIM_Q2D) {
            aA = al * v.Area[c];
            rq = 1.0 / (1.0 - aA * (-g1 * vv));
        }
    }
    // field e of the padded list: X fields first (NGX groups), then C (NGC groups)
    auto field = [&](int e) -> double {
        if (!ok) return 0.0;
        if (e < NGX * G) return e < D ? v.Dq[e * N + c] : 0.0;
        const int m = e - NGX * G;
        if (m == F::AL) return al;
        if (m == F::AA) return aA;
        if (m == F::RQ) return rq;
        if (m == F::G1) return g1;
        if (m < F::Y) return hvs + v.DHi[(m - F::DP) * N + c];
        if (m < F::U) return v.w[(4 + m - F::Y) * N + c];
        if (m == F::U) return u;
        if (m == F::V) return vv;
        if (m == F::H) return v.w[(D + 2) * N + c];
        if (m < F::PB) return dir[0][m - F::PA];
        if (m < F::NC) return dir[1][m - F::PB];
        return 0.0;
    };
    const long long s0 = step_off[b.x] + kPadSteps + b.y;
    T* outX = X + s0 * L::XS;
    T* outC = Cr + s0 * L::CS;
    const int nt = min(32, ni + 31 - b.y);
    using V = typename Vec16<T>::type;
    // the fields of the next two groups are loaded before this group's barrier
    // and transpose, so that their global loads overlap it
    T cur[G], nxt[G], nx2[G];
#pragma unroll
    for (int e = 0; e < G; ++e) {
        cur[e] = T(field(e));
        nxt[e] = T(field(G + e));
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
            T* dst = g < NGX ? outX + (long long)wt * L::XS + g * 32 * G : outC + (long long)wt * L::CS + (g - NGX) * 32 * G;
            *reinterpret_cast<V*>(dst + wl * G) = *reinterpret_cast<V*>(vals);
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
struct WaveArgs {
    const int4* tasks;          // (plane, first strip, strips, forward index of the plane's strip 0)
    int ntasks;
    const long long* step_off;  // per forward strip: first step block of its records (padding included)
    void* X;
    void* C;
    void* xfer;                 // per task: its published hand-off columns
    long long xstride;          // elements per task
    int* progress;              // per task: hand-off chunks published
    int* ticket;
};

namespace {

__device__ __forceinline__ void give_up(const View& v, int* s_bail) {
    *reinterpret_cast<volatile int*>(s_bail) = 1;
    atomicExch(&v.sc->spin_abort, 1ull);
    atomicMax(&v.sc->status, SCFD_E_SPIN);
}
__device__ __forceinline__ bool aborted(const View& v, const int* s_bail) {
    return *reinterpret_cast<const volatile int*>(s_bail) != 0 ||
           *reinterpret_cast<const volatile unsigned long long*>(&v.sc->spin_abort) != 0ull;
}
// bounded wait on a phase of a local mbarrier.  Every phase these kernels wait
// for completes on the waiting CTA's own barrier (bulk-copy transaction counts,
// or arrivals that carry no data the waiter reads), so CTA-scope acquire is
// enough.
__device__ __forceinline__ bool wait_phase(unsigned long long* bar, unsigned par, const View& v, const int* s_bail) {
    // a phase that has already completed is seen by the non-blocking test
    // cheaper than by try_wait (about 50 cycles less per wait in the sweeps)
    if (mbar_test_wait(bar, par)) return true;
    long long spins = 0;
    while (!mbar_try_wait(bar, par)) {
        if (++spins > kSpin || ((spins & 1023) == 0 && aborted(v, s_bail))) return false;
    }
    return true;
}

}  // namespace

// one CTA per SM (its shared memory); the bound lets ptxas use the registers that
// leaves (FP64 146-162, FP32 102-112, no spill; FP64 sweep pair 0.856 -> 0.837 ms)
template <typename RT, int NY, int DIR>
__global__ void __cluster_dims__(CL, 1, 1) __launch_bounds__(64, 1) k_wave(View v, WaveArgs a) {
    using F = CF<NY>;
    using L = WL<RT, NY>;
    using V = typename Vec16<RT>::type;
    constexpr int D = NY + 3, G4 = L::G, NGX = L::NGX, NGC = L::NGC, XS = L::XS, CSZ = L::CS, D4 = L::D4,
                  SPB = L::SPB, PFB = L::PFB;
    constexpr unsigned CHUNK_BYTES = HK * D4 * sizeof(RT);
    static_assert(SPB <= kPadSteps, "a record chunk may reach into the padding by at most one chunk");
    static_assert(D4 % G4 == 0 && (CHUNK_BYTES % 16) == 0, "hand-off chunks are whole 16-byte vectors");
    extern __shared__ __align__(128) unsigned char sm[];
    RT* ringX = reinterpret_cast<RT*>(sm);   // [PFB][SPB][XS]
    RT* ringC = ringX + PFB * SPB * XS;      // [PFB][SPB][CS]
    RT* xin = ringC + PFB * SPB * CSZ;       // [HS][HK][D4]: columns from the strip below
    RT* xout = xin + HS * HK * D4;           // [HS][HK][D4]: top row for the next task (via the helper)
    unsigned long long* bars = reinterpret_cast<unsigned long long*>(xout + HS * HK * D4);
    unsigned long long* rfull = bars;          // record slot loaded (helper: expect_tx + bulk copies)
    unsigned long long* rdone = bars + PFB;    // record slot computed (compute warp arrive)
    unsigned long long* xfull = bars + 2 * PFB;  // hand-off chunk arrived (producer's arrival + bytes)
    unsigned long long* pempty = xfull + HS;   // successor consumed a chunk this CTA produced
    unsigned long long* hempty = pempty + HS;  // this CTA consumed a chunk its helper fetched
    unsigned long long* oful = hempty + HS;    // xout chunk written (compute lane 31)
    unsigned long long* oemp = oful + HS;      // xout chunk published (helper)
    int* s_task = reinterpret_cast<int*>(oemp + HS);
    int* s_bail = s_task + 1;

    __shared__ __align__(16) RT s_zero[D4];  // the strip-below column where there is none
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned rank = cluster_rank();
    if (sizeof(RT) == 8 && threadIdx.x < D4) s_zero[threadIdx.x] = RT(0);
    if (threadIdx.x == 0) {
        for (int k = 0; k < 2 * PFB + 5 * HS; ++k) mbar_init(&bars[k], 1);
        *s_bail = 0;
        *s_task = 0;
        mbar_init_fence();
    }
    __syncthreads();
    cluster_sync();

    const bool q2d = v.dim == SCFD_DIM_Q2D;
    // running uses (over all tasks of this cluster) of this CTA's rings
    unsigned rc = 0;  // record chunks
    unsigned xc = 0;  // hand-off chunks consumed from xin
    unsigned pc = 0;  // chunks of this CTA's top row produced through xout

    for (;;) {
        if (threadIdx.x == 0 && rank == 0) {
            int t = atomicAdd(a.ticket, 1);
            if (aborted(v, s_bail)) t = a.ntasks;
            *s_task = t;
        }
        cluster_sync();
        int task;
        {
            const unsigned ra = mapa(s_task, 0);
            asm volatile("ld.shared::cluster.s32 %0, [%1];" : "=r"(task) : "r"(ra) : "memory");
        }
        if (task >= a.ntasks) break;
        const int4 tk = a.tasks[task];
        const int p = tk.x, s0 = tk.y, ns = tk.z, fsb = tk.w;
        const int ni = v.P.ni[p], nstr = (v.P.nj[p] + 31) / 32;
        const bool active = (int)rank < ns;
        const int strip = DIR == 0 ? s0 + (int)rank : s0 - (int)rank;
        const int fs = fsb + strip;
        const bool pred_task = DIR == 0 ? s0 > 0 : s0 < nstr - 1;
        const bool succ_task = DIR == 0 ? s0 + ns < nstr : s0 - ns >= 0;
        const bool has_prev = active && (rank > 0 || pred_task);
        const bool pub_remote = active && (int)rank + 1 < ns;
        const bool pub_global = active && (int)rank + 1 == ns && succ_task;
        const int nsteps = ni + 31;
        const int nch = (nsteps + SPB - 1) / SPB;
        const int nxc = chunks_of(ni);
        const long long sbase = active ? a.step_off[fs] + kPadSteps : 0;
        // first record step (memory order) of chunk n
        auto chunk_step = [&](int n) -> long long {
            return DIR == 0 ? (long long)n * SPB : (long long)(ni + 30) - (long long)n * SPB - (SPB - 1);
        };

        if (warp == 0 && active) {
            // ------------------------------------------------------------ compute warp
            bool bail = false;
            const int lf = DIR == 0 ? lane : 31 - lane;  // this lane's slot in a step block
            // consumed chunks are released to the producer: the CTA below (remote) or this CTA's helper
            const unsigned rel = rank > 0 ? mapa(pempty, rank - 1) : mapa(hempty, rank);
            // the next CTA's hand-off ring and its barriers (pub_remote)
            const unsigned dring = pub_remote ? mapa(xin, rank + 1) : 0u;
            const unsigned dfull = pub_remote ? mapa(xfull, rank + 1) : 0u;
            RT outA[D], outB[D];
#pragma unroll
            for (int k = 0; k < D; ++k) {
                outA[k] = RT(0);
                outB[k] = RT(0);
            }
            // The hand-off.  Chunk j of the strip below holds the columns 4j-3 .. 4j
            // (HK = 4) of its top row: its lane 31 computes column c at its step c + 31,
            // so its group of steps G (4G .. 4G+3) yields exactly chunk G - 7.  Lane 0
            // here uses column t at step t: chunk G's last column at step 4G (u = 0 of
            // group G), chunk G+1's first three at u = 1..3, so chunk G is released and
            // chunk G+1 awaited between u = 0 and u = 1.
            static_assert(HK == 4 && SPB % HK == 0, "groups of 4 steps, whole groups per record slot");
            const int lastc = nxc - 1;
            const unsigned xc0 = xc;
            unsigned xw = xc;  // chunks awaited (running, like xc)
            auto await_chunk = [&]() -> bool {
                const bool ok = wait_phase(&xfull[xw % HS], (xw / HS) & 1u, v, s_bail);
                ++xw;
                return __all_sync(0xffffffffu, ok);
            };
            if (has_prev && !await_chunk()) {
                if (lane == 0) give_up(v, s_bail);
                bail = true;
            }
            for (int n = 0; n < nch && !bail; ++n) {
                const unsigned slot = rc % PFB, par = (rc / PFB) & 1u;
                if (!__all_sync(0xffffffffu, wait_phase(&rfull[slot], par, v, s_bail))) {
                    if (lane == 0) give_up(v, s_bail);
                    bail = true;
                    break;
                }
                RT* sx = ringX + slot * SPB * XS;
                const RT* scf = ringC + slot * SPB * CSZ;
#pragma unroll
                for (int h = 0; h < SPB / HK && !bail; ++h) {
                    const int G = n * (SPB / HK) + h;
                    // this group's top-row outputs form chunk J of the strip above
                    const int J = G - 7;
                    const bool pub = (pub_remote || pub_global) && J >= 0 && J <= lastc;
                    const unsigned ps = pc % HS;
                    // back-pressure once per 8 chunks: chunk pc + k (k < 8) reuses the
                    // slot of chunk pc + k - HS, and chunks are released in order, so
                    // the release of chunk pc + 7 - HS covers the next 8
                    if (pub && pc % 8u == 0u && pc + 7u >= HS) {
                        const unsigned pw = pc + 7u, sw = pw % HS;
                        const bool okp =
                            wait_phase(pub_remote ? &pempty[sw] : &oemp[sw], ((pw / HS) - 1u) & 1u, v, s_bail);
                        if (!__all_sync(0xffffffffu, okp)) {
                            if (lane == 31) give_up(v, s_bail);
                            bail = true;
                            break;
                        }
                    }
#pragma unroll
                    for (int u = 0; u < HK; ++u) {
                        const int t = G * HK + u;
                        const int pos = DIR == 0 ? h * HK + u : SPB - 1 - (h * HK + u);
                        if (u == 1 && has_prev) {
                            // chunk G is used up; chunk G+1 holds the next three columns.  A
                            // chunk is refilled HS chunks later, long after these reads.
                            if (G <= lastc) {
                                if (lane == 0) mbar_arrive_cluster_relaxed(rel + (xc % HS) * 8u);
                                ++xc;
                            }
                            if (G + 1 <= lastc && !await_chunk()) {
                                if (lane == 0) give_up(v, s_bail);
                                bail = true;
                                break;
                            }
                        }
                        // column t from the strip below (lane 0)
                        // Where there is no strip below or the column is past the plane,
                        // the FP64 step reads a zero column (one address select instead of a
                        // value select per component: FP64 sweep pair 0.879 -> 0.850 ms); the
                        // FP32 step keeps the value selects, which measured faster for it
                        // (0.578 against 0.592 ms).
                        const bool in_col = has_prev && t < ni;
                        const RT* xring = xin + (((xc0 + (unsigned)((t + 3) >> 2)) % HS) * HK + ((t + 3) & 3)) * D4;
                        const RT* xi = sizeof(RT) == 8 && !in_col ? s_zero : xring;
                        // every lane reads the column (16-byte shared-memory broadcasts); lane 0 uses it
                        RT xv[D4];
#pragma unroll
                        for (int g = 0; g < D4 / G4; ++g)
                            *reinterpret_cast<V*>(&xv[g * G4]) = reinterpret_cast<const V*>(xi)[g];
                        RT inB[D];
#pragma unroll
                        for (int k = 0; k < D; ++k) {
                            const RT sh = __shfl_up_sync(0xffffffffu, outB[k], 1);
                            if constexpr (sizeof(RT) == 8)
                                inB[k] = lane == 0 ? xv[k] : sh;
                            else
                                inB[k] = lane == 0 ? (in_col ? xv[k] : RT(0)) : sh;
                        }
                        // this lane's cell
                        RT fx[NGX * G4], f[NGC * G4];
                        const V* srcx = reinterpret_cast<const V*>(sx + pos * XS) + lf;
                        const V* srcc = reinterpret_cast<const V*>(scf + pos * CSZ) + lf;
#pragma unroll
                        for (int g = 0; g < NGX; ++g) *reinterpret_cast<V*>(&fx[g * G4]) = srcx[g * 32];
#pragma unroll
                        for (int g = 0; g < NGC; ++g) *reinterpret_cast<V*>(&f[g * G4]) = srcc[g * 32];
                        const RT al = f[F::AL];
                        RT x[D];
#pragma unroll
                        for (int k = 0; k < D; ++k)
                            x[k] = DIR == 0 ? al * (fx[k] + (outA[k] + inB[k])) : fx[k] - al * (outA[k] + inB[k]);
                        // dpdq (sch_NR.raw.f90:143-144): species hvs + DHi (from the record),
                        // then -g1 u, -g1 v, g1
                        const RT g1 = f[F::G1], uu = f[F::U], vv = f[F::V];
                        RT dp[D];
#pragma unroll
                        for (int k = 0; k < NY; ++k) dp[k] = f[F::DP + k];
                        dp[NY] = -g1 * uu;
                        dp[NY + 1] = -g1 * vv;
                        dp[NY + 2] = g1;
                        // P = dpdq.x; forward q2d: semi-implicit pressure source
                        // (q2d time_lusgs_viscous.f90:38-44).  Both sums are pairwise trees.
                        RT pr[D - 1];
#pragma unroll
                        for (int k = 0; k < D - 1; ++k) {
                            const int kk = k < NY + 1 ? k : k + 1;  // every component but rho v
                            pr[k] = dp[kk] * x[kk];
                        }
                        RT P = tree_sum<0, D - 1>(pr);
                        const RT S = tree_sum<0, NY>(x);
                        if (DIR == 0 && q2d) x[NY + 1] = (x[NY + 1] + f[F::AA] * P) * f[F::RQ];
                        P += dp[NY + 1] * x[NY + 1];
#pragma unroll
                        for (int dn = 0; dn < 2; ++dn) {
                            // ds/2 folded into the direction's coefficients (k_pack):
                            // o = (Y, u, v, H) fb + (fa lam) x + (fa n1, fa n2, fa un) P
                            const int b0 = dn == 0 ? F::PA : F::PB;
                            const RT p1 = f[b0 + F::P1], p2 = f[b0 + F::P2], pu = f[b0 + F::PU];
                            const RT fl = f[b0 + (DIR == 0 ? F::LP : F::LM)];
                            const RT fb = p1 * x[NY] + p2 * x[NY + 1] - pu * S;
                            RT* o = dn == 0 ? outA : outB;
#pragma unroll
                            for (int k = 0; k < NY; ++k) o[k] = f[F::Y + k] * fb + fl * x[k];
                            o[NY] = uu * fb + fl * x[NY] + p1 * P;
                            o[NY + 1] = vv * fb + fl * x[NY + 1] + p2 * P;
                            o[NY + 2] = f[F::H] * fb + fl * x[NY + 2] + pu * P;
                        }
                        // results back into the slot (16-byte stores); the helper writes them out
#pragma unroll
                        for (int k = 0; k < D; ++k) fx[k] = x[k];
                        V* dstx = reinterpret_cast<V*>(sx + pos * XS) + lf;
#pragma unroll
                        for (int g = 0; g < NGX; ++g) dstx[g * 32] = *reinterpret_cast<V*>(&fx[g * G4]);
                        // lane 31: entry u of chunk J in this CTA's xout ring
                        if (pub && lane == 31) {
                            RT vals[D4];
#pragma unroll
                            for (int k = 0; k < D4; ++k) vals[k] = k < D ? outB[k] : RT(0);
                            RT* dst = xout + (ps * HK + u) * D4;
#pragma unroll
                            for (int g = 0; g < D4 / G4; ++g)
                                reinterpret_cast<V*>(dst)[g] = *reinterpret_cast<V*>(&vals[g * G4]);
                        }
                    }
                    if (bail) break;
                    // chunk J complete: one bulk copy into the next CTA's ring, completing the
                    // receiver's barrier phase with this arrival and the copy's bytes (in
                    // either order), or on to the helper, which publishes it in global
                    // memory.  Columns outside 0 .. ni-1 travel as they are.
                    if (pub) {
                        if (lane == 31) {
                            fence_proxy_async_smem();
                            if (pub_remote) {
                                mbar_arrive_expect_tx_cluster_relaxed(dfull + ps * 8u, CHUNK_BYTES);
                                bulk_s2dsmem(dring + ps * CHUNK_BYTES, xout + ps * HK * D4, CHUNK_BYTES, dfull + ps * 8u);
                            } else {
                                mbar_arrive(&oful[ps]);
                            }
                        }
                        ++pc;
                    }
                }
                if (bail) break;
                // the slot's results are visible to the helper's bulk store
                fence_proxy_async_smem();
                __syncwarp();
                if (lane == 0) mbar_arrive(&rdone[slot]);
                ++rc;
            }
        } else if (warp == 1 && active) {
            // ------------------------------------------------------------ helper warp
            RT* gX = reinterpret_cast<RT*>(a.X) + sbase * XS;
            const RT* gC = reinterpret_cast<const RT*>(a.C) + sbase * CSZ;
            const bool gin = rank == 0 && pred_task;
            const int* prog_in = a.progress + (task > 0 ? task - 1 : 0);
            int* prog_out = a.progress + task;
            const RT* xsrc = reinterpret_cast<const RT*>(a.xfer) + (long long)(task > 0 ? task - 1 : 0) * a.xstride;
            RT* xdst = reinterpret_cast<RT*>(a.xfer) + (long long)task * a.xstride;
            const unsigned rc0 = rc, xc0 = xc, pc0 = pc;
            int nl = 0, nst = 0, hin = 0, hout = 0;
            long long idle = 0;
            bool bail = false;
            while (!bail && (nst < nch || (gin && hin < nxc) || (pub_global && hout < nxc))) {
                bool prog = false;
                // record loads: the slot of chunk nl is free once chunk nl - PFB is stored
                if (nl < nch && nl - PFB < nst) {
                    if (lane == 0) {
                        if (nl >= PFB) bulk_wait_read_all();
                        const unsigned slot = (rc0 + nl) % PFB;
                        const long long st0 = chunk_step(nl);
                        mbar_expect_tx(&rfull[slot], SPB * (XS + CSZ) * sizeof(RT));
                        tma_bulk_g2s(ringX + slot * SPB * XS, gX + st0 * XS, SPB * XS * sizeof(RT), &rfull[slot]);
                        tma_bulk_g2s(ringC + slot * SPB * CSZ, gC + st0 * CSZ, SPB * CSZ * sizeof(RT), &rfull[slot]);
                    }
                    ++nl;
                    prog = true;
                }
                // results of computed chunks back to X
                if (nst < nl) {
                    const unsigned slot = (rc0 + nst) % PFB;
                    int done = 0;
                    if (lane == 0) done = mbar_test_wait(&rdone[slot], ((rc0 + nst) / PFB) & 1u) ? 1 : 0;
                    if (__shfl_sync(0xffffffffu, done, 0)) {
                        if (lane == 0) {
                            tma_bulk_s2g(gX + chunk_step(nst) * XS, ringX + slot * SPB * XS, SPB * XS * sizeof(RT));
                            bulk_commit();
                        }
                        ++nst;
                        prog = true;
                    }
                }
                // hand-off columns of the task below, through global memory
                if (gin && hin < nxc) {
                    const unsigned g = xc0 + hin, hs = g % HS;
                    int go = 0;
                    if (lane == 0) {
                        const bool free = g < HS || mbar_test_wait(&hempty[hs], ((g / HS) - 1u) & 1u);
                        if (free && ld_acquire_gpu(prog_in) >= hin + 1) {
                            fence_proxy_async_global();
                            mbar_expect_tx(&xfull[hs], CHUNK_BYTES);
                            tma_bulk_g2s(xin + hs * HK * D4, xsrc + (long long)hin * HK * D4, CHUNK_BYTES, &xfull[hs]);
                            go = 1;
                        }
                    }
                    if (__shfl_sync(0xffffffffu, go, 0)) {
                        ++hin;
                        prog = true;
                    }
                }
                // this task's top row, published to the task above
                if (pub_global && hout < nxc) {
                    const unsigned g = pc0 + hout, hs = g % HS;
                    int rd = 0;
                    if (lane == 0) rd = mbar_test_wait(&oful[hs], (g / HS) & 1u) ? 1 : 0;
                    if (__shfl_sync(0xffffffffu, rd, 0)) {
                        for (int e = lane; e < HK * D4; e += 32) xdst[(long long)hout * HK * D4 + e] = xout[hs * HK * D4 + e];
                        __threadfence();
                        __syncwarp();
                        if (lane == 0) {
                            st_release_gpu(prog_out, hout + 1);
                            mbar_arrive(&oemp[hs]);
                        }
                        ++hout;
                        prog = true;
                    }
                }
                if (prog) {
                    idle = 0;
                } else if (++idle > kSpin || ((idle & 1023) == 0 && aborted(v, s_bail))) {
                    if (lane == 0) give_up(v, s_bail);
                    bail = true;
                }
            }
            // loads issued but never consumed (after a bail) land before the slot is reused or the CTA exits
            if (lane == 0) {
                for (int n = nst; n < nl; ++n) {
                    const unsigned slot = (rc0 + n) % PFB;
                    long long spins = 0;
                    while (!mbar_try_wait(&rfull[slot], ((rc0 + n) / PFB) & 1u) && ++spins < kSpin) {
                    }
                }
                bulk_wait_read_all();
            }
            __syncwarp();
            rc = rc0 + nch;
            if (gin) xc = xc0 + nxc;
            if (pub_remote || pub_global) pc = pc0 + nxc;
        }
        cluster_sync();  // the task is done in every CTA of the cluster
    }
    if (warp == 1 && lane == 0) bulk_wait_all();
    __syncwarp();
    cluster_sync();  // no CTA leaves while a peer may still reach its shared memory
}

// ---------------------------------------------------------------------------
// k_omega: the NR relaxation's candidates from the backward sweep's result
// (time_NR_viscous.f90:56-78): per block of 32 steps x 32 lanes of a strip,
// res = sum of Dq(E)^2 and omega = min over Dq_k < 0 of -q_k / Dq_k * Dqmax,
// into partials[2 b], partials[2 b + 1].  Records are read coalesced (step y,
// lane x) and turned to cells (step x, lane y) through shared memory, so that
// q is read along rows.
// ---------------------------------------------------------------------------
template <typename T, int NY>
__global__ void __launch_bounds__(1024) k_omega(View v, const int2* blk, const int4* strips, const long long* step_off,
                                                const T* X, double* partials) {
    using L = WL<T, NY>;
    constexpr int G = L::G;
    __shared__ double tile[32][33];
    const int2 b = blk[blockIdx.x];
    const int4 st = strips[b.x];
    const int p = st.x, s = st.y;
    const int ni = v.P.ni[p], nj = v.P.nj[p];
    const T* in = X + (step_off[b.x] + kPadSteps + b.y) * L::XS;
    const int nt = min(32, ni + 31 - b.y);
    const long long N = v.ncell;
    const bool rd = (int)threadIdx.y < nt;
    const long long rbase = (long long)threadIdx.y * L::XS + threadIdx.x * G;
    const int tt = threadIdx.x, l = threadIdx.y;
    const int t = b.y + tt, cc = t - l, j = 32 * s + 1 + l;
    const bool wr = tt < nt && cc >= 0 && cc < ni && j <= nj;
    const long long c = wr ? cidx(v.P, p, cc + 1, j) : 0;
    double res = 0.0, om = 1e300;
    // every record value and q of the block's cells are loaded before the first
    // barrier, so that the loads overlap one another instead of one component's
    // barriers
    double xr[NY + 1], qr[NY];
#pragma unroll
    for (int m = 0; m <= NY; ++m) {
        const int k = m < NY ? m : NY + 2;  // the species, then the energy
        xr[m] = rd ? double(in[rbase + (long long)(k / G) * 32 * G + k % G]) : 0.0;
    }
#pragma unroll
    for (int m = 0; m < NY; ++m) qr[m] = wr ? v.q[m * N + c] : 0.0;
#pragma unroll
    for (int m = 0; m <= NY; ++m) {
        tile[threadIdx.y][threadIdx.x] = xr[m];
        __syncthreads();
        if (wr) {
            const double dq = tile[tt][l];
            if (m < NY) {
                if (dq < 0.0) om = fmin(om, -qr[m] / dq * v.dq_max);
            } else {
                res = dq * dq;
            }
        }
        __syncthreads();
    }
    double* out = partials + 2 * blockIdx.x;
    // the block's cells in a fixed order: warps, then lanes
    for (int d = 16; d > 0; d >>= 1) {
        res += __shfl_down_sync(0xffffffffu, res, d);
        om = fmin(om, __shfl_down_sync(0xffffffffu, om, d));
    }
    if (threadIdx.x == 0) {
        tile[0][threadIdx.y] = res;
        tile[1][threadIdx.y] = om;
    }
    __syncthreads();
    if (threadIdx.y == 0) {
        res = tile[0][threadIdx.x];
        om = tile[1][threadIdx.x];
        for (int d = 16; d > 0; d >>= 1) {
            res += __shfl_down_sync(0xffffffffu, res, d);
            om = fmin(om, __shfl_down_sync(0xffffffffu, om, d));
        }
        if (threadIdx.x == 0) {
            out[0] = res;
            out[1] = om;
        }
    }
}

// ---------------------------------------------------------------------------
// k_unpack: q += omega * Dq from the records (LU-SGS: omega = 1; NR: the
// positivity-limited omega reduced from k_omega's per-block partials in fixed order,
// time_NR_viscous.f90:86-108).
// ---------------------------------------------------------------------------
template <typename T, int NY>
__global__ void __launch_bounds__(1024) k_unpack(View v, const int2* blk, const int4* strips, const long long* step_off,
                                                 const T* X, const double* partials, int nstrips, int nr_mode,
                                                 int inner) {
    using L = WL<T, NY>;
    constexpr int D = NY + 3, G = L::G;
    __shared__ double tile[32][33];
    double om = 1.0;
    if (nr_mode) {
        // every block reduces the partials alike (fixed order)
        double res, o;
        reduce_partials(partials, nstrips, res, o);
        if (blockIdx.x == 0 && threadIdx.x == 0 && threadIdx.y == 0) {
            if (o < v.omega_min) atomicMax(&v.sc->status, SCFD_E_OMEGA);
            if (inner == 1) v.sc->res1 = res;
            v.sc->res = res;
            v.sc->omega = fmin(v.omega_max, o);
            log_inner(v.sc, inner, o, res);
        }
        // time_NR_viscous.f90:75-78: below omega_min the step stops without the update
        if (o < v.omega_min || v.sc->status == SCFD_E_OMEGA) return;
        om = fmin(v.omega_max, o);
    }
    const int2 b = blk[blockIdx.x];
    const int4 st = strips[b.x];
    const int p = st.x, s = st.y;
    const int ni = v.P.ni[p], nj = v.P.nj[p];
    const T* in = X + (step_off[b.x] + kPadSteps + b.y) * L::XS;
    const int nt = min(32, ni + 31 - b.y);
    const long long N = v.ncell;
    // read (step y, lane x) coalesced, write cells (step x, lane y); every record
    // value and q of the block's cells are loaded before the first barrier, so
    // that the loads overlap one another
    const bool rd = (int)threadIdx.y < nt;
    const long long rbase = (long long)threadIdx.y * L::XS + threadIdx.x * G;
    const int tt = threadIdx.x, l = threadIdx.y;
    const int t = b.y + tt, cc = t - l, j = 32 * s + 1 + l;
    const bool wr = tt < nt && cc >= 0 && cc < ni && j <= nj;
    const long long c = wr ? cidx(v.P, p, cc + 1, j) : 0;
    double xr[D], qr[D];
#pragma unroll
    for (int k = 0; k < D; ++k) xr[k] = rd ? double(in[rbase + (long long)(k / G) * 32 * G + k % G]) : 0.0;
#pragma unroll
    for (int k = 0; k < D; ++k) qr[k] = wr ? v.q[k * N + c] : 0.0;
#pragma unroll
    for (int k = 0; k < D; ++k) {
        if (rd) tile[threadIdx.y][threadIdx.x] = xr[k];
        __syncthreads();
        if (wr) v.q[k * N + c] = nr_mode ? qr[k] + om * tile[tt][l] : qr[k] + tile[tt][l];
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
int wave_pad_steps() { return kPadSteps; }
int wave_strips_per_task() { return CL; }
int wave_handoff_chunk() { return HK; }
int wave_chunks(int ni) { return chunks_of(ni); }

namespace {
template <typename RT, int NY>
WaveSizes sizes_t() {
    using L = WL<RT, NY>;
    return WaveSizes{L::XS, L::CS, L::D4, L::SMEM};
}
}  // namespace

WaveSizes wave_sizes(int ny, bool mixed) {
    switch (ny) {
        case 1: return mixed ? sizes_t<float, 1>() : sizes_t<double, 1>();
        case 8: return mixed ? sizes_t<float, 8>() : sizes_t<double, 8>();
        case 9: return mixed ? sizes_t<float, 9>() : sizes_t<double, 9>();
        default: return WaveSizes{0, 0, 0, 0};
    }
}

namespace {

template <typename RT, int NY, int DIR>
int max_clusters_t() {
    using L = WL<RT, NY>;
    if (cudaFuncSetAttribute(k_wave<RT, NY, DIR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L::SMEM) !=
        cudaSuccess)
        return 0;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(CL, 1, 1);
    cfg.blockDim = dim3(64, 1, 1);
    cfg.dynamicSmemBytes = L::SMEM;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = CL;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    // the kernel carries its cluster shape; some runtimes want it repeated
    // in the query's attributes, others reject that
    int n = 0;
    cfg.numAttrs = 0;
    if (cudaOccupancyMaxActiveClusters(&n, k_wave<RT, NY, DIR>, &cfg) == cudaSuccess && n > 0) return n;
    cudaGetLastError();
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, k_wave<RT, NY, DIR>, &cfg) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

template <typename RT, int NY>
int max_clusters_ny() {
    const int f = max_clusters_t<RT, NY, 0>(), b = max_clusters_t<RT, NY, 1>();
    return f < b ? f : b;
}

}  // namespace

int wave_max_clusters(int ny, bool mixed) {
    switch (ny) {
        case 1: return mixed ? max_clusters_ny<float, 1>() : max_clusters_ny<double, 1>();
        case 8: return mixed ? max_clusters_ny<float, 8>() : max_clusters_ny<double, 8>();
        case 9: return mixed ? max_clusters_ny<float, 9>() : max_clusters_ny<double, 9>();
        default: return 0;
    }
}

namespace {

template <typename RT, int NY, int DIR>
void sweep_launch(const View& v, cudaStream_t s, const Wave& w) {
    using L = WL<RT, NY>;
    WaveArgs a{DIR == 0 ? w.tasks_f : w.tasks_b, w.ntasks,    w.step_off, w.X, w.C, w.xfer, w.xstride,
               w.progress + (DIR == 0 ? 0 : w.ntasks), w.tickets + (DIR == 0 ? 0 : 1)};
    const int ncl = w.nclusters < w.ntasks ? w.nclusters : w.ntasks;
    k_wave<RT, NY, DIR><<<ncl * CL, 64, L::SMEM, s>>>(v, a);
}

template <typename RT, int NY>
void run_t(const View& v, cudaStream_t s, const Wave& w, int what, int inner) {
    const bool nr = v.scheme == SCFD_SCHEME_NR;
    if (what == 0) {
        k_pack<RT, NY><<<w.nblk, dim3(32, 32), 0, s>>>(v, w.blk, w.strips, w.step_off, reinterpret_cast<RT*>(w.X),
                                                       reinterpret_cast<RT*>(w.C), nr ? 1 : 0);
    } else if (what == 3) {
        k_unpack<RT, NY><<<w.nblk, dim3(32, 32), 0, s>>>(v, w.blk, w.strips, w.step_off,
                                                         reinterpret_cast<const RT*>(w.X), w.partials, w.nstrips,
                                                         nr ? 1 : 0, inner);
    } else if (what == 4) {
        k_omega<RT, NY><<<w.nblk, dim3(32, 32), 0, s>>>(v, w.blk, w.strips, w.step_off,
                                                        reinterpret_cast<const RT*>(w.X), w.partials);
    } else if (what == 1) {
        sweep_launch<RT, NY, 0>(v, s, w);
    } else {
        sweep_launch<RT, NY, 1>(v, s, w);
    }
}

}  // namespace

// what: 0 pack, 1 forward sweep, 2 backward sweep, 3 unpack/update, 4 the NR
// partials (res, omega) of the backward sweep's result
int launch_wave(const View& v, cudaStream_t s, const Wave& w, int what, int inner) {
    const bool mixed = v.precision == SCFD_PREC_MIXED;
    switch (v.nY) {
        case 1: if (mixed) run_t<float, 1>(v, s, w, what, inner); else run_t<double, 1>(v, s, w, what, inner); return 1;
        case 8: if (mixed) run_t<float, 8>(v, s, w, what, inner); else run_t<double, 8>(v, s, w, what, inner); return 1;
        case 9: if (mixed) run_t<float, 9>(v, s, w, what, inner); else run_t<double, 9>(v, s, w, what, inner); return 1;
        default: return 0;
    }
}

}  // namespace scfd
