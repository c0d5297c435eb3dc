// scfd_internal.h -- device data layout and kernel interfaces of the B200
// path.  Everything here is private to libscfd_b200.so.
//
// Layout in HBM (one arena per context):
//   * A "cell slot" index c addresses cell (i,j) of plane p for i = -1..ni+2,
//     j = -1..nj+2 (two ghost layers, as q(.., -1:nimax+2, -1:njmax+2, ..)):
//         c = base[p] + (j + 1) * pitch[p] + (i + 1),
//     pitch[p] = round_up(ni + 4, 32) so rows start on 256-byte boundaries;
//     a plane holds nj + 4 rows.
//     Planes follow each other; all planes are resident together.
//   * Every field is structure-of-arrays: component k of field F lives at
//     F[k * ncell + c].  Face quantities of face i+1/2 (resp. j+1/2) are stored
//     in the slot of cell i (resp. j), so dsi(i,j) -> dsi[c(i,j)].
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/scfd_b200.h"

namespace scfd {

constexpr int kMaxPlanes = SCFD_MAX_PLANES;
constexpr int kMaxSpecies = SCFD_MAX_SPECIES;

struct Planes {
    int np;
    int ni[kMaxPlanes];
    int nj[kMaxPlanes];
    int pitch[kMaxPlanes];
    long long base[kMaxPlanes];
    // planes this context updates (all of them unless the case is sharded over
    // ranks); kernels with one grid row per plane run over act[0..nact)
    int nact;
    int act[kMaxPlanes];
};

__host__ __device__ inline long long cidx(const Planes& P, int p, int i, int j) {
    return P.base[p] + (long long)(j + 1) * P.pitch[p] + (i + 1);
}

// Per-species contribution lists of the reaction rates, in the order in which
// the reference accumulates them.  For Fex_var (FJ.f90:301-453) entry 2*i + kind
// adds the forward (kind 0) or reverse (kind 1) rate of reaction i; p lists the
// production terms, m the destruction terms; mref[i] is the reaction whose
// third-body term reaction i uses (-1: none yet).  For Fex / Jex
// (FJ.f90:152-709), the net list of species j, n_ptr[j] .. n_ptr[j+1], holds
// 2*i + 1 for every reactant slot of j in reaction i and 2*i for every product
// slot, reactions in order and reactants first, as the reference subtracts and
// adds Dr; dref[i] is the last reaction up to i that sets dlnkdlnM (third-body
// or fall-off rate; -1: none yet).
struct RateLists {
    const int* p_ptr;  // [ns+1]
    const int* p_ent;
    const int* m_ptr;  // [ns+1]
    const int* m_ent;
    const int* mref;   // [nr]
    const int* n_ptr;  // [ns+1]
    const int* n_ent;
    const int* dref;   // [nr]
};

// Compact chemistry tables on the device (0-based species).
struct DevChem {
    int ns, nr, nt;
    const double* coeff;      // [ns][2][7]
    const double* tcommon;    // [ns] Tthre(3,k)
    const double* inv_mw;     // [ns] 1/MW (computed as 1d0/MWs like invMW)
    const double* mws;        // [ns]
    const int* rstate;        // [nr][2]
    const int* indnu;         // [nr][2][3]
    const int* numnu;         // [nr][2]
    const int* snu;           // [nr]
    const int* exist_m;       // [nr]
    const int* numm;          // [nr]
    const int* indm;          // [nr][ns]
    const double* men;        // [nr][ns]
    const double* abe;        // [nr][3]
    const double* cabe;       // [nr][3]
    const double* troe;       // [nr][4]
    const int* tr2th;         // [nt]
    const int* nsec;          // [nt]
    const double* trange;     // [nt][5][2]
    const double* trans;      // [nt][5][4]
    const double* wc1;        // [nt][nt] (MW(jt)/MW(it))**0.25
    const double* wc2;        // [nt][nt] sqrt(2 MW(jt)/(MW(it)+MW(jt)))
    RateLists rl;             // the per-species rate lists of the one-warp evaluations
    double rtol, atol;        // control_chem.inp tolerances (atol: DVODE only)
};

// Scalars that live on the device between kernels of one step.
struct DevScalars {
    double dt_grbl;
    double tt;
    double omega;          // omega applied by the last NR update
    double res;            // last inner residual
    double res1;           // first inner residual of the step
    unsigned long long dtmin_bits;  // atomicMin target for the global dt
    int status;            // SCFD_* code, atomicMax
    int first_dual;
    long long chem_attempts;
    long long chem_fallback;
    long long chem_attempts_last;  // the same counts for the last chemistry launch only
    long long chem_fallback_last;
    unsigned long long spin_abort;  // non-zero once a bounded wait gave up
    // per inner iteration of the last step (internal_res.dat of
    // time_NR_viscous.f90:87-95): omega from the Dqrate limiter before the
    // omega_max cap, and the residual sum
    double il_omega[SCFD_INNER_LOG];
    double il_res[SCFD_INNER_LOG];
};
// records the inner iteration's omega candidate and residual (inner >= 1)
__device__ __forceinline__ void log_inner(DevScalars* sc, int inner, double omega_raw, double res) {
    if (inner >= 1 && inner <= SCFD_INNER_LOG) {
        sc->il_omega[inner - 1] = omega_raw;
        sc->il_res[inner - 1] = res;
    }
}

// (res, omega) of n partials (pairs), reduced by every thread of a block of
// up to 1024 threads in a fixed order (the same value in every block and every
// run): res summed, omega the minimum.  Every thread of the block must call it.
__device__ __forceinline__ void reduce_partials(const double* part, int n, double& res, double& om) {
    __shared__ double s_r[32], s_o[32];
    const int tid = (threadIdx.z * blockDim.y + threadIdx.y) * blockDim.x + threadIdx.x;
    const int nth = blockDim.x * blockDim.y * blockDim.z;
    const int lane = tid & 31, wid = tid >> 5, nw = (nth + 31) >> 5;
    double r = 0.0, o = 1e300;
    for (int k = tid; k < n; k += nth) {
        r += part[2 * k];
        o = fmin(o, part[2 * k + 1]);
    }
    for (int d = 16; d > 0; d >>= 1) {
        r += __shfl_down_sync(0xffffffffu, r, d);
        o = fmin(o, __shfl_down_sync(0xffffffffu, o, d));
    }
    __syncthreads();  // s_r / s_o may still be read by a previous call
    if (lane == 0) {
        s_r[wid] = r;
        s_o[wid] = o;
    }
    __syncthreads();
    if (wid == 0) {
        r = lane < nw ? s_r[lane] : 0.0;
        o = lane < nw ? s_o[lane] : 1e300;
        for (int d = 16; d > 0; d >>= 1) {
            r += __shfl_down_sync(0xffffffffu, r, d);
            o = fmin(o, __shfl_down_sync(0xffffffffu, o, d));
        }
        if (lane == 0) {
            s_r[0] = r;
            s_o[0] = o;
        }
    }
    __syncthreads();
    res = s_r[0];
    om = s_o[0];
}

// All device pointers of a context; passed by value to the kernels.
struct View {
    Planes P;
    long long ncell;
    int nY, D, W;
    int dim, viscous, recon, thermo, mu_model, scheme, dt_mode, precision;
    double phi_mus, k_mus, kappa, rgas, nu_gas, suth_mu0, suth_t0, suth_s, prandtl, schmidt, cfl, dt_fixed;
    double omega_max, omega_min, dq_max;
    double cfl_tau;              // DUAL: pseudo-time CFL
    // launch shapes chosen by the autotuner (scfd_api.cu::autotune)
    int res_tile;                // index into residual2_tiles()
    int thermo_block;            // threads per CTA of k_thermo (64, 128 or 256)
    // state
    double *q, *qp, *qpp, *w, *vhi, *DHi, *Dq, *dt_mat;
    double *alpha, *nuA, *nuB;   // LU-SGS coefficients per cell
    double* pre;                 // DUAL: pre_sca(1..4) per cell, pre[k * ncell + c]
    // geometry
    double *Vol, *Area, *dsi, *dsj, *vni, *vnj, *x, *r, *gjc, *gji, *gjj, *dsci, *dscj, *vnci, *vncj;
    // mixed-precision copies used by the FP32 residual / sweeps
    float *w32, *vhi32;
    double* base;  // arena base: every double field above is base + a whole offset
    DevScalars* sc;
    DevChem chem;
};

// One ghost-cell write of set_BC (halo copy or boundary descriptor).
struct GhostOp {
    long long dst;   // ghost cell slot
    long long src;   // interior cell slot read
    int kind;        // -1 halo copy, else SCFD_BC_*
    int bc;          // descriptor index for values
    double n1, n2;   // boundary face normal (SLIP)
};

// kernels / launchers (stream-ordered); each returns the number of launches
int launch_thermo(const View& v, cudaStream_t s, int cells_per_plane_max);
int launch_ghosts(const View& v, cudaStream_t s, const GhostOp* ops, int nops, const double* bcval, int valstride);
int launch_ghost_ops(const View& v, cudaStream_t s, const GhostOp* ops, int nops, const double* bcval, int valstride);
int launch_set_dt(const View& v, cudaStream_t s);
int launch_set_dt_cells(const View& v, cudaStream_t s);  // dt_mat and the local minimum only
int launch_residual(const View& v, cudaStream_t s, int mode, bool need_coeffs);
bool launch_residual2(const View& v, cudaStream_t s, int mode);
int residual2_tiles(int* tx, int* ty);  // the tile shapes of k_residual2 (count; tx, ty may be null)
int launch_sweep_reset(cudaStream_t s, int* progress, int* tickets, int nstrips_fwd, int nstrips_bwd);
int launch_sweep(const View& v, cudaStream_t s, int dir, double* xfer, int* progress, double* partials,
                 int* tickets, int nstrips_fwd, int nstrips_bwd, const int* strip_tab_f, const int* strip_tab_b);
bool launch_sweep2(const View& v, cudaStream_t s, int dir, const int2* strips, int n, double* xfer, int* prog,
                   int* ticket, double* partials, int upd);
// Cluster-wavefront LU-SGS over strip records (k_wave.cu), for nY in {1, 8, 9}.
struct Wave {
    void* X;                    // records: x(1:D) per cell and step (float on the mixed path)
    void* C;                    // records: the cells' coefficients
    const long long* step_off;  // per forward strip: first step block of its records
    const int4* strips;         // per forward strip (plane, s, strip, 0): pack / unpack
    const int2* blk;            // pack/unpack blocks: (strip, first step)
    int nblk;
    int nstrips;
    const int4* tasks_f;        // tasks of up to 8 strips (plane, first strip, strips, strip 0's index)
    const int4* tasks_b;        // backward order
    int ntasks;
    int nclusters;              // clusters launched (at most ntasks)
    void* xfer;                 // per task: published hand-off columns
    long long xstride;          // elements per task
    int* progress;              // 2*ntasks
    int* tickets;               // 2
    double* partials;           // (res, omega) per pack block: 2*nstrips, nstrips = nblk
};
struct WaveSizes {
    int xs, cs, d4;  // elements of an X / C step block; padded hand-off column
    size_t smem;     // dynamic shared memory of the sweep kernel
};
WaveSizes wave_sizes(int ny, bool mixed);  // xs = 0 if the species count has no sweep
int wave_pad_steps();                      // zero step blocks before and after each strip
int wave_strips_per_task();
int wave_handoff_chunk();                  // hand-off columns per chunk
int wave_chunks(int ni);                   // hand-off chunks of a top row of ni columns
int wave_max_clusters(int ny, bool mixed); // co-resident clusters of the sweep kernel (0: none)
int launch_wave(const View& v, cudaStream_t s, const Wave& w, int what, int inner);
int launch_nr_update(const View& v, cudaStream_t s, const double* partials, int nstrips, int inner);
// Cells whose CHEMEQ2 interval went to DVODE: k_chem queues them (the cell, the
// time reached and the moles and T there) and k_chem_dvode finishes them.
struct ChemQueue {
    long long* cell;             // [capacity]
    double* tt;                  // [capacity]
    double* y;                   // [capacity][ns + 1]
    unsigned long long* count;   // 2: queued, taken
    long long capacity;          // interior cells of the updated planes
    int warp_doubles;            // shared memory per warp of k_chem_dvode
    int warps_per_block;
};
size_t chem_dvode_warp_doubles(int ns, int nr);
int chem_dvode_setup(int ns, int nr, int* warps_per_block);  // kernel attribute; 0 or a cudaError_t
int launch_chem_impl(const View& v, cudaStream_t s, int max_substeps, unsigned long long* counter, int nsm,
                     const ChemQueue& dq);
int launch_step_end(const View& v, cudaStream_t s, double warn, double err);
int launch_rms(const View& v, cudaStream_t s, double* partial, double* out);
int launch_copy(double* dst, const double* src, long long n, cudaStream_t s);
int launch_scalar_begin(const View& v, cudaStream_t s);
int launch_to_f32(const View& v, cudaStream_t s);
// reference layout <-> SoA slots (dir 0: ref -> soa, dir 1: soa -> ref_out)
int launch_ref_soa(const View& v, cudaStream_t s, int nk, int IX, int JX, const double* ref, double* soa,
                   double* ref_out, int dir);

// block sharding (k_shard.cu): exchange of the cells other ranks' ghost
// copies read, and the device halves of the cross-rank reductions
struct HaloImport {
    long long slot;  // cell written
    long long off;   // buffer index of component 0
    long long n;     // buffer stride between components
};
int launch_halo_pack(const View& v, cudaStream_t s, const long long* cells, int n, double* out);
int launch_halo_unpack(const View& v, cudaStream_t s, const HaloImport* imp, int n, const double* buf);
int launch_dt_export(const View& v, cudaStream_t s, double* red);        // red = [dt_min, -status]
int launch_dt_import(const View& v, cudaStream_t s, const double* red);
int launch_res_export(const View& v, cudaStream_t s, const double* partials, int nstrips, double* red);
int launch_res_import(const View& v, cudaStream_t s, const double* red, int inner);  // red = [res, omega, -status]
int launch_status_export(const View& v, cudaStream_t s, double* red);    // red = [-status]
int launch_status_import(const View& v, cudaStream_t s, const double* red);

// discrete adjoint of the explicit ideal-gas step (k_adjoint.cu)
int launch_adj_faces(const View& v, cudaStream_t s, const double* lam, double* wbar, double dt);
int launch_adj_ghost(const View& v, cudaStream_t s, const GhostOp* ops, int nops, const double* bcval, int valstride,
                     double* wbar, double* grad, int param_bc);
int launch_adj_prim(const View& v, cudaStream_t s, double* wbar, double* lam);
int launch_adj_objective(const View& v, cudaStream_t s, const long long* cells, const double* wt, int n, double* J,
                         double* lam, int grad_only);

// residual modes (RES_DUAL: NR's right-hand side multiplied by Gamma^-1 and the
// coefficients of the preconditioned dual time; RES_PRECON / RES_PRECON_LUSGS:
// the preconditioned local time step, spectral radii and alpha of the precon
// schemes and their right-hand side multiplied by I + phh p1 p2^T)
enum { RES_EULER = 0, RES_LUSGS = 1, RES_NR = 2, RES_DUAL = 3, RES_PRECON = 4, RES_PRECON_LUSGS = 5 };

// NR, the preconditioned dual time and precon share the dual-time main loop
__host__ __device__ inline bool dual_time_scheme(int scheme) {
    return scheme == SCFD_SCHEME_NR || scheme == SCFD_SCHEME_DUAL || scheme == SCFD_SCHEME_PRECON;
}
// the two schemes of time_scheme/precon and time_scheme/preconLU-SGS
__host__ __device__ inline bool precon_scheme(int scheme) {
    return scheme == SCFD_SCHEME_PRECON || scheme == SCFD_SCHEME_PRECON_LUSGS;
}

}  // namespace scfd
