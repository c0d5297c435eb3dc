/*
 * scfd_b200.h -- C ABI of the B200 (sm_100a) implementation of shared_cfd's
 * per-step residual-and-implicit-update path.
 *
 * The reference has no plugin or FFI layer.  Its "operator API" is the set of
 * fixed subroutine names that the generated main.f90 calls every step
 * (store/core/main.part_primitive.f90:2-3, store/core/main.part_main.f90:2-5,
 * store/time_scheme/<scheme>/main.main*.f90) plus the module-global arrays of
 * store/core/variable.f90:1-49.  A Fortran architecture variant binds the
 * functions below with iso_c_binding and replaces that call sequence with one
 * scfd_step() per physical step; everything between upload and download stays
 * resident on the GPU.
 *
 * Conventions
 *   - Every function returns an int status (SCFD_OK == 0).  Nothing aborts the
 *     process; the reference's `stop` / `call exit(1)` sites become codes.
 *   - Plane, cell and species indices in descriptors are 1-based, like the
 *     reference's Fortran.
 *   - Field arrays crossing the ABI use the reference's own layout, e.g.
 *     q(1:dimq,-1:nimax+2,-1:njmax+2,1:Nplane) in Fortran column-major order,
 *     so a Fortran caller passes its module arrays unchanged.
 *   - A context owns all device memory and one CUDA stream.  It is not
 *     thread-safe; use one context per host thread / GPU.
 */
#ifndef SCFD_B200_H
#define SCFD_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SCFD_ABI_VERSION 1

#define SCFD_MAX_PLANES    64
#define SCFD_MAX_SPECIES   32
#define SCFD_MAX_REACTIONS 256
#define SCFD_MAX_TRANS_SEC 5
/* w(1:dimw) followed by vhi(1:nY): dimw = nY+8 */
#define SCFD_BC_MAXVAL     (2 * SCFD_MAX_SPECIES + 8)

/* ---- status codes ------------------------------------------------------ */
enum {
    SCFD_OK             = 0,
    SCFD_E_ARG          = 1,  /* bad argument / descriptor                        */
    SCFD_E_CUDA         = 2,  /* CUDA runtime error                               */
    SCFD_E_TNEWTON      = 3,  /* T-from-e Newton exceeded max_T_loop (sub_chem.f90:1575-1579) */
    SCFD_E_CHEM         = 4,  /* chemistry integrator did not converge (sub_chem.f90:1767,1812) */
    SCFD_E_OMEGA        = 5,  /* NR relaxation omega < omega_min (NR/q2d/time_NR_viscous.f90:75-78) */
    SCFD_E_RESRATE      = 6,  /* inner residual ratio > ResRateErr (NR/q2d/sch_NR.raw.f90:232-233) */
    SCFD_E_NAN          = 7,  /* NaN in the RMS of rho*E (core/check_convergence.f90:29-32) */
    SCFD_E_SPIN         = 8,  /* a bounded device wait gave up (wavefront flag)   */
    SCFD_E_CONNECT      = 9,  /* bad connectivity record                          */
    SCFD_E_IO           = 10, /* file input / output                              */
    SCFD_E_STATE        = 11, /* call out of order (e.g. step before commit)      */
    SCFD_E_UNSUPPORTED  = 12, /* option combination not provided                 */
    SCFD_E_SINGULAR     = 13  /* CEA Newton matrix singular twice in one cell: the
                                 reference stops the program (NASA/core/sub_chem.f90:1472-1488) */
};

/* ---- option enums (values follow checkout.inp where one exists) ------- */
enum { SCFD_DIM_2D = 0, SCFD_DIM_Q2D = 1 };                   /* checkout_flow.py:105-118 */
enum { SCFD_DT_GLOBAL = 0, SCFD_DT_LOCAL = 1, SCFD_DT_FIXED = 2 }; /* checkout_flow.py:120-132; FIXED: dt given */
/* checkout_flow.py:134-181 (the values of its time-scheme line); DUAL is the
 * Weiss-Smith preconditioned dual time of store/time_scheme/dual/2d (2d, global
 * or fixed dt, non-reacting: checkout_flow.py:159-168) */
enum {
    SCFD_SCHEME_EULER = 0,
    SCFD_SCHEME_LUSGS = 2,
    SCFD_SCHEME_NR = 3,
    SCFD_SCHEME_PRECON = 4,        /* time_scheme/precon/2d: preconditioned NR inner loop, local dt */
    SCFD_SCHEME_DUAL = 5,
    SCFD_SCHEME_PRECON_LUSGS = 6   /* time_scheme/preconLU-SGS/2d: preconditioned LU-SGS, local dt */
};
enum { SCFD_RECON_UPWIND = 0, SCFD_RECON_MUSCL = 1 };           /* checkout_flow.py:183-194 */
enum { SCFD_THERMO_IDEAL = 0, SCFD_THERMO_CHEMKIN_COLD = 1, SCFD_THERMO_CHEMKIN_REACTIVE = 2 };
enum { SCFD_MU_REFERENCE = 0, SCFD_MU_SUTHERLAND = 1 };        /* ideal gas viscosity law */
enum { SCFD_PREC_FP64 = 0, SCFD_PREC_MIXED = 1 };

/* Boundary kinds for the device boundary descriptors.  They cover the ghost
 * fills written by hand in the sample condition.f90 files (e.g.
 * sample/no27.chemkin_reaction/condition.f90:49-147); ghost layer 2 always
 * copies ghost layer 1, as in those samples. */
enum {
    SCFD_BC_EXTRAP    = 0,  /* zero gradient: ghost = first interior cell            */
    SCFD_BC_FIXED     = 1,  /* ghost w(1:dimw), vhi(1:nY) = value[]                   */
    SCFD_BC_OUTFLOW_P = 2,  /* zero gradient, then w(4) = value[0]                    */
    SCFD_BC_SLIP      = 3,  /* zero gradient, velocity mirrored about the face normal */
    SCFD_BC_NOSLIP    = 4,  /* zero gradient, u,v -> 2*value[0..1] - u,v (adiabatic)   */
    SCFD_BC_FIXED_PIN = 5   /* fixed state w(1:dimw), vhi(1:nY) = value[], except
                               p = interior p and rho = (p*value[dimw+nY]) /
                               value[dimw+nY+1], the inflow of
                               sample/no27.chemkin_reaction/condition.f90:49-60   */
};
enum { SCFD_SIDE_ILO = 0, SCFD_SIDE_IHI = 1, SCFD_SIDE_JLO = 2, SCFD_SIDE_JHI = 3 };

/* ---- descriptors ------------------------------------------------------- */
typedef struct scfd_desc {
    int32_t abi_version;           /* = SCFD_ABI_VERSION                          */
    int32_t nplane;                /* Nplane (store/core/n_grid.raw.f90:4)        */
    int32_t ni[SCFD_MAX_PLANES];   /* cells per plane in i                        */
    int32_t nj[SCFD_MAX_PLANES];   /* cells per plane in j                        */
    int32_t ny;                    /* nY: species count (1 for ideal gas)         */
    int32_t dim;                   /* SCFD_DIM_*                                  */
    int32_t dt_mode;               /* SCFD_DT_*                                   */
    int32_t scheme;                /* SCFD_SCHEME_*                               */
    int32_t recon;                 /* SCFD_RECON_*                                */
    int32_t viscous;               /* 0 non-viscous, 1 viscous (no-nV variant)    */
    int32_t thermo;                /* SCFD_THERMO_*                               */
    int32_t mu_model;              /* SCFD_MU_* (ideal gas only)                  */
    int32_t precision;             /* SCFD_PREC_*                                 */
    int32_t quirk_q1;              /* 1: reproduce geometry.f90:95-103 whole-array
                                      ghost extrapolation (reference behaviour)   */
    int32_t num_internal_loop;     /* NR "InternalLoop Max Number" (N-1 inner its)*/
    int32_t il_write;              /* NR "InternalLoop OutOmega" (diagnostic only)*/
    double  phi_mus, k_mus;        /* MUSCL parameters (muscl.f90:87-106)         */
    double  kappa, rgas, nu_gas;   /* ideal gas KAPPA, RGAS, NU (checkout_flow.py:216-221) */
    double  suth_mu0, suth_t0, suth_s; /* Sutherland law (mu_model = SUTHERLAND)  */
    double  prandtl, schmidt;      /* reference: Pr = Sc = 1 (sch_viscous.f90:98-99) */
    double  cfl;                   /* control.inp "CFL Number"                    */
    double  dt_fixed;              /* dt for SCFD_DT_FIXED                        */
    double  omega_max, omega_min, dq_max, res_rate_warn, res_rate_err; /* NR control */
    int32_t chem_max_substeps;     /* device cap on chemistry substeps per cell   */
    int32_t pad0;
    double  cfl_tau;               /* DUAL: control.inp "InternalLoop CFL tau" (> 0) */
    int32_t reserved[12];
} scfd_desc;

typedef struct scfd_bc {
    int32_t plane;                 /* 1-based                                     */
    int32_t side;                  /* SCFD_SIDE_*                                 */
    int32_t first, last;           /* inclusive cell range along the side         */
    int32_t kind;                  /* SCFD_BC_*                                   */
    int32_t pad;
    double  value[SCFD_BC_MAXVAL + 2];
} scfd_bc;

/* Chemkin tables after parsing chem.inp / MW.inp / trans.inp and the
 * fuel/oxidiser species reordering (store/therm_lib/chemkin/core/mod_chem.raw.f90:31-68,
 * sub_chem.f90:191-502, 788-889, 968-979).  Species indices are 0-based here. */
typedef struct scfd_chem {
    int32_t ns, nr, nt;
    int32_t pad0;
    double  coeff[SCFD_MAX_SPECIES][2][7];   /* coeff(i,sec,k) -> [k][sec-1][i-1]  */
    double  tthre[SCFD_MAX_SPECIES][3];
    double  mws[SCFD_MAX_SPECIES];
    int32_t rstate[SCFD_MAX_REACTIONS][2];
    int32_t indnu[SCFD_MAX_REACTIONS][2][3];
    int32_t numnu[SCFD_MAX_REACTIONS][2];
    int32_t snu[SCFD_MAX_REACTIONS];
    int32_t exist_m[SCFD_MAX_REACTIONS];
    int32_t numm[SCFD_MAX_REACTIONS];
    int32_t indm[SCFD_MAX_REACTIONS][SCFD_MAX_SPECIES];
    double  men[SCFD_MAX_REACTIONS][SCFD_MAX_SPECIES];
    double  abe[SCFD_MAX_REACTIONS][3];      /* (ln A, beta, Ea/Rc)                */
    double  cabe[SCFD_MAX_REACTIONS][3];
    double  troe[SCFD_MAX_REACTIONS][4];
    int32_t tr2th[SCFD_MAX_SPECIES];         /* transport entry -> species (0-based) */
    int32_t num_sctn_trans[SCFD_MAX_SPECIES];
    double  trange_trans[SCFD_MAX_SPECIES][SCFD_MAX_TRANS_SEC][2];
    double  trans[SCFD_MAX_SPECIES][SCFD_MAX_TRANS_SEC][4];
    double  rtol, atol;                      /* control_chem.inp tolerances        */
} scfd_chem;

/* inner iterations recorded per step by scfd_inner_log */
#define SCFD_INNER_LOG 128

typedef struct scfd_stats {
    double  dt_grbl;               /* global dt of the step (global / fixed mode) */
    double  tt;                    /* accumulated physical time                   */
    double  res, res1;             /* NR: last and first inner residual sums      */
    double  omega;                 /* NR: last relaxation factor applied          */
    int32_t status;                /* SCFD_* code of the step                     */
    int32_t inner_iters;           /* NR inner iterations run                     */
    int64_t chem_attempts;         /* CHEMEQ2 attempts summed over cells          */
    int64_t chem_fallback_cells;   /* cells that used the implicit fallback       */
    int32_t res_warn;              /* 1 if res/res1 > ResRateWarn                 */
    int32_t reserved[7];
} scfd_stats;

typedef struct scfd_ctx scfd_ctx;

/* ---- lifecycle ---------------------------------------------------------- */
int  scfd_abi_version(void);
/* Replaces the compile-time sizing of store/core/n_grid.raw.f90 and the
 * checkout.inp selections (store/checkout/checkout_flow.py:67-327). */
int  scfd_create(const scfd_desc* desc, scfd_ctx** out);
int  scfd_destroy(scfd_ctx* ctx);
/* Error text of the last failing call on this context. */
int  scfd_last_error(const scfd_ctx* ctx, char* buf, int len);

/* ---- set-up ------------------------------------------------------------- */
/* Node coordinates of one plane, xh(0:ni,0:nj), rh(0:ni,0:nj), column-major
 * (store/dim/2d/geometry.f90:27-78, init_xrh). */
int  scfd_set_geometry(scfd_ctx* ctx, int plane, const double* xh, const double* rh);
/* Block-interface records, 11 ints each, exactly the lines of cut_copro000.inp
 * (geo width order p1 c1 s1 pm1 p2 c2 s2 pm2; store/cond/core/mod_cond.py:271-276,
 * consumed by section_exchange, store/cond/no-nV/condition.tail.f90:2-70). */
int  scfd_set_connectivity(scfd_ctx* ctx, const int32_t* recs, int nrec);
/* Device boundary descriptors replacing the user loops of set_BC. */
int  scfd_set_bc(scfd_ctx* ctx, const scfd_bc* bcs, int nbc);
/* Chemkin tables (required for SCFD_THERMO_CHEMKIN_*). */
int  scfd_set_chem(scfd_ctx* ctx, const scfd_chem* chem);
/* Ends set-up: builds the metrics (init_geometry, set_vnc_dsc, set_geojac),
 * allocates device memory and checks the connectivity. */
int  scfd_commit(scfd_ctx* ctx);

/* ---- state -------------------------------------------------------------- */
/* q(1:dimq,-1:nimax+2,-1:njmax+2,Nplane), w(1:dimw,...), vhi(1:nY,...):
 * the reference's module arrays (store/core/variable.f90:24-33).  vhi may be
 * NULL (then it is computed by scfd_prepare).  qp/qpp are set to q. */
int  scfd_upload(scfd_ctx* ctx, const double* q, const double* w, const double* vhi,
                 double tt);
/* part_primitive (set_w, set_thermo_prop) followed by set_BC(step):
 * store/core/main.body.raw.f90:15-16. */
int  scfd_prepare(scfd_ctx* ctx, int step);
/* One physical step of the configured scheme, the body of the generated time
 * loop (store/time_scheme/<scheme>/main.main*.f90 with part_* expanded). */
int  scfd_step(scfd_ctx* ctx, int step, scfd_stats* stats);
/* nsteps consecutive calls of scfd_step starting at step; stats of the last. */
int  scfd_run(scfd_ctx* ctx, int step, int nsteps, scfd_stats* stats);
/* RMS of check_convergence (store/core/check_convergence.f90:17-28):
 * sqrt(sum (q(E)-qp(E))^2) / ncells over all planes. */
int  scfd_rms(scfd_ctx* ctx, double* rms);
/* The inner-iteration record of the last NR / dual / precon step, as the
 * reference writes internal_res.dat with "InternalLoop OutOmega"
 * (store/time_scheme/NR/q2d/time_NR_viscous.f90:87-95): for inner iteration
 * k = 1..n, omega[k-1] is the relaxation factor from the Dqrate limiter before
 * the omega_max cap (1e300 when no species decreases) and res[k-1] the residual
 * sum (res/res1 is the reference's third column).  Writes min(n, inner
 * iterations of the step, SCFD_INNER_LOG) entries and returns that count (< 0:
 * an SCFD_E_* code, negated).  Either pointer may be NULL. */
int  scfd_inner_log(scfd_ctx* ctx, double* omega, double* res, int n);
/* Copies the state back in the reference layout; any pointer may be NULL. */
int  scfd_download(scfd_ctx* ctx, double* q, double* w, double* vhi, double* tt);
/* Same as download but for qp (the previous step's q). */
int  scfd_download_qp(scfd_ctx* ctx, double* qp);
/* restart.bin / result/result<step>.bin of out_bin (store/core/inout.f90:1-75):
 * three Fortran sequential-unformatted big-endian records, the step (int32),
 * tt (float64) and, for every plane, j = 0..nj+1, i = 0..ni+1 (i fastest),
 * q(1:dimq), w(indxR), w(indxg), w(4).  Before the field is taken the first
 * ghost layer of q is recomputed from w as set_bc_q does (inout.f90:144-200),
 * in the written copy only.  SCFD_E_IO if the file cannot be written. */
int  scfd_write_restart(scfd_ctx* ctx, const char* path, int step);
/* restart_bin (inout.f90:77-100): reads such a file into q and w(indxR),
 * w(indxg), w(4) of cells i = 0..ni+1, j = 0..nj+1 (the rest of the state is
 * kept), sets tt and qp = qpp = q as scfd_upload does, and returns the step.
 * SCFD_E_IO for a missing, truncated or mis-sized file.  After commit. */
int  scfd_read_restart(scfd_ctx* ctx, const char* path, int* step, double* tt);
/* geometry.bin of out_geo_bin (store/dim/2d/geometry.f90:182-193): per plane
 * the records ni, nj (int32) and (xh, rh) of nodes i = 0..ni, j = 0..nj
 * (i fastest), big-endian.  After scfd_set_geometry of every plane. */
int  scfd_write_geometry(scfd_ctx* ctx, const char* path);
/* The context's CUDA stream (cudaStream_t as void*), for event timing. */
int  scfd_get_stream(scfd_ctx* ctx, void** stream);
/* Number of device kernel launches issued by the last scfd_step/scfd_run. */
int  scfd_launch_count(const scfd_ctx* ctx, int64_t* count);

/* Per-kernel timing.  While enabled, every kernel of a step is bracketed by
 * CUDA events on the context's stream and its device time accumulated per
 * kind; scfd_kernel_stats reads (and scfd_profile(ctx,1) resets) the totals. */
enum {
    SCFD_K_THERMO = 0, SCFD_K_BC, SCFD_K_DT, SCFD_K_CHEM, SCFD_K_RESIDUAL,
    SCFD_K_SWEEP_FWD, SCFD_K_SWEEP_BWD, SCFD_K_UPDATE, SCFD_K_COPY, SCFD_K_OTHER, SCFD_K_PACK,
    SCFD_K_COUNT
};
int  scfd_profile(scfd_ctx* ctx, int enable);
/* The launch shapes the autotuner picked for this context, as a JSON object
 * (residual tile shape, thermo CTA size, the device time of every candidate).
 * The tuner runs once per context, before its first step: each candidate is
 * timed with CUDA events on the context's own state (saved before and
 * restored after) and the fastest is kept; the candidates compute the same
 * values.  SCFD_AUTOTUNE=0 in the environment keeps the default shapes;
 * SCFD_RES_TILE=<k> pins the residual to tile k of the list (e.g. to profile
 * one shape). */
int  scfd_tuning(scfd_ctx* ctx, char* json, int len);
int  scfd_kernel_stats(scfd_ctx* ctx, int kind, double* total_ms, int64_t* launches, char* name, int namelen);

/* ---- discrete adjoint of the explicit ideal-gas step ------------------------
 * The reference has no adjoint.  For a 2d inviscid ideal-gas case on the
 * explicit Euler scheme with a fixed dt (FP64), scfd_adjoint_run runs nsteps
 * physical steps from the uploaded state and returns
 *   J = sum over steps n in [win_first, win_last] of
 *       sum over the boundary cells of descriptor obj_bc of ds * p(q^n)
 * (the pressure force on that boundary: p of the first interior cell times the
 * boundary face length) and dJ/dvalue of descriptor param_bc's values (the
 * inflow state of a SCFD_BC_FIXED descriptor, for instance), by the reverse of
 * every step: the MUSCL + SLAU residual, the ghost writes and the primitive
 * map, hand-differentiated (the branches of SLAU's min / max / abs as taken
 * forward).  States are recomputed from at most `snapshots` stored ones by
 * binomial checkpointing.  counts (may be NULL) receives the forward and the
 * reverse steps taken.  On return the context holds the uploaded state again.
 * Other configurations return SCFD_E_UNSUPPORTED. */
typedef struct scfd_adj_desc {
    int32_t abi_version;
    int32_t nsteps;              /* physical steps, >= 1                           */
    int32_t snapshots;           /* stored states besides the initial one, >= 0  */
    int32_t obj_bc;              /* 0-based descriptor index of the objective     */
    int32_t win_first, win_last; /* 0 <= win_first <= win_last < nsteps           */
    int32_t param_bc;            /* 0-based descriptor of the gradient, -1: none  */
    int32_t forward_only;        /* 1: J only                                     */
    int32_t reserved[8];
} scfd_adj_desc;
/* grad: SCFD_BC_MAXVAL + 2 doubles, one per value[] entry of param_bc. */
int  scfd_adjoint_run(scfd_ctx* ctx, const scfd_adj_desc* desc, double* J, double* grad, int64_t* counts);
/* Replaces the value[] of boundary descriptor bc (0-based) after commit. */
int  scfd_set_bc_values(scfd_ctx* ctx, int bc, const double* value);

/* ---- block-sharded step over several processes (one GPU each) -------------
 * Replaces the MPI decomposition of the reference: the cross-rank halo copies
 * of set_BC (store/cond/no-nV/condition.tail.f90:71-330, MPI_Isend/Recv of w
 * and vhi) and the reductions of dt_grbl (store/time_step/global/set_dt.f90:40),
 * of omega and the inner residual (store/time_scheme/NR/q2d/time_NR_viscous.f90:
 * 87-90, here reduced to every rank: quirk Q4 off) and of the RMS
 * (store/core/check_convergence.f90:33).  Every rank holds the whole case, all
 * planes, and updates only the planes `owner` gives it.  LU-SGS needs no
 * exchange (Dq = 0 at plane edges).
 *
 * The library communicates nothing itself.  A sharded physical step is a
 * sequence of scfd_dstep calls; each enqueues the work up to the next point
 * where the ranks must agree and returns a request that the caller fulfils on
 * req->buf (device memory of the context's stream on the CUDA library, host
 * memory on the CPU restatement) before the next call:
 *   SCFD_DREQ_REDUCE  all-reduce SUM of buf[0..nsum) and MIN of
 *                     buf[nsum..nsum+nmin); a status travels as -status in a
 *                     MIN slot, so the MIN is the worst status
 *   SCFD_DREQ_HALO    all-gather: buf is nranks segments of seg doubles; this
 *                     rank's segment is filled, the others must hold their
 *                     ranks' segments on return
 *   SCFD_DREQ_DONE    the step is complete; the return value is the step's
 *                     status (the same on every rank) and stats is filled
 * Every rank issues the same requests in the same order, whatever the status.
 * Work on the CUDA library stays on the context's stream (scfd_get_stream);
 * the caller orders its collectives on that stream.  In stats,
 * chem_attempts and chem_fallback_cells count this rank's cells; dt, time,
 * res, res1 and omega are global.  scfd_rms returns this rank's share,
 * sqrt(sum over owned cells)/(all cells): the global RMS is the square root of
 * the sum of the ranks' squares.  scfd_download returns all planes, of which
 * only the owned ones are current. */
#define SCFD_MAX_RANKS 64
enum { SCFD_DREQ_DONE = 0, SCFD_DREQ_REDUCE = 1, SCFD_DREQ_HALO = 2 };
typedef struct scfd_dreq {
    int32_t kind;     /* SCFD_DREQ_* */
    int32_t nsum;     /* REDUCE: leading slots summed */
    int32_t nmin;     /* REDUCE: following slots minimised */
    int32_t nranks;   /* HALO: segments */
    int64_t seg;      /* HALO: doubles per segment */
    double* buf;
} scfd_dreq;
/* Before scfd_commit: owner[p] (0-based rank, p = 0..nplane-1) of every plane,
 * the number of ranks and this rank.  A context without a partition owns every
 * plane and may also step through scfd_dstep (as rank 0 of 1). */
int  scfd_set_partition(scfd_ctx* ctx, const int32_t* owner, int nranks, int rank);
/* Begins or continues a sharded physical step.  scfd_step and scfd_run refuse
 * a context partitioned over more than one rank (SCFD_E_STATE). */
int  scfd_dstep(scfd_ctx* ctx, int step, scfd_dreq* req, scfd_stats* stats);

/* ---- batched constant-volume 0-D reactors ---------------------------------
 * Replaces per-reactor calls of reaction_chemeq2 / reaction_one_steps
 * (store/therm_lib/chemkin/core/sub_chem.f90:1684-1713 and 1396-1504).  Each
 * reactor integrates its moles n_1..n_ns (mol/cm^3, from the partial densities
 * as n = vrho/MW*1e-3, floored at 1e-40) and T from t = 0 to t_end by
 * successive reaction_chemeq2 calls over dt_call (CHEMEQ2, sub_chem.f90:1714-1819,
 * on the UV source terms; each call starts its own attempt count and floors n
 * at 1e-40 on entry and exit, as the reference's), and records the ignition
 * delay of reaction_one_steps (sub_chem.f90:1467-1472): the first time
 * T >= T0 + dT_ign, interpolated linearly between the accepted substeps around
 * it (the state at t = 0 is the first of them).  Where the reference hands the
 * rest of a call to DVODE after 10 CHEMEQ2 attempts, the library takes
 * two-stage Rosenbrock (ROS2) substeps on Fex and its exact Jacobian Jex
 * (FJ.f90:152-300, 454-709, the pair the reference hands DVODE) and flags the reactor
 * SCFD_REACTOR_FELL_BACK. */
enum {
    SCFD_REACTOR_QUEUE = 0,      /* one persistent launch, reactors drawn from a device work queue
                                    (replayed from a CUDA graph after the first run) */
    SCFD_REACTOR_PER_LAUNCH = 1  /* one kernel launch per reactor */
};
enum { SCFD_REACTOR_IGNITED = 1, SCFD_REACTOR_FELL_BACK = 2, SCFD_REACTOR_FAILED = 4 };

typedef struct scfd_reactor_desc {
    int32_t abi_version;
    int32_t n;             /* reactors in this run (<= n_max of scfd_reactors_create) */
    int32_t mode;          /* SCFD_REACTOR_QUEUE / SCFD_REACTOR_PER_LAUNCH */
    int32_t max_substeps;  /* accepted substeps per call before SCFD_E_CHEM (<= 0: 1e6) */
    double  t_end;         /* s */
    double  dT_ign;        /* K (the reference uses 400) */
    double  dt_call;       /* s: interval of each reaction_chemeq2 call (a flow solver's
                              time step); <= 0 means one call over [0, t_end] */
    int32_t reserved[6];
} scfd_reactor_desc;

typedef struct scfd_reactors scfd_reactors;

int   scfd_reactors_create(const scfd_chem* chem, int n_max, scfd_reactors** out);
int   scfd_reactors_destroy(scfd_reactors* r);
/* T0[n] in K; vrho0[n][ns] partial densities in kg/m^3 (the q(1:ns) of a cell) */
int   scfd_reactors_upload(scfd_reactors* r, int n, const double* T0, const double* vrho0);
/* integrates the uploaded reactors, asynchronously on scfd_reactors_stream(r) */
int   scfd_reactors_launch(scfd_reactors* r, const scfd_reactor_desc* d);
/* after a launch: T_end[n], vrho_end[n][ns], t_ign[n] (s, -1 when T never
 * reached T0 + dT_ign), evals[n] = source-term (Fex_var) evaluations (2 per
 * CHEMEQ2 attempt, 2 per Rosenbrock substep: one Jex, one Fex), flags[n]; any pointer may be
 * NULL.  Returns the worst status of the run. */
int   scfd_reactors_download(scfd_reactors* r, double* T_end, double* vrho_end, double* t_ign, int64_t* evals,
                             int32_t* flags);
/* upload + launch + download */
int   scfd_reactors_run(scfd_reactors* r, const scfd_reactor_desc* d, const double* T0, const double* vrho0,
                        double* T_end, double* vrho_end, double* t_ign, int64_t* evals, int32_t* flags);
void* scfd_reactors_stream(scfd_reactors* r);
/* kernel launches made by the last scfd_reactors_launch */
int   scfd_reactors_launch_count(const scfd_reactors* r, int64_t* launches);

/* ---- chemical source terms and their Jacobian -------------------------- */
/* Fex and Jex (store/therm_lib/chemkin/uvhp/uv/FJ.f90:152-300 and 454-709), the
 * right-hand side and exact Jacobian the reference hands DVODE, for n states
 * at once on the device.  states[n][ns+1] = (n_1..n_ns in mol/cm^3, T in K);
 * dndt[n][ns+1] receives the net rates and dT/dt at constant volume;
 * jac[n][ns+1][ns+1] (row-major, d dndt_i / d state_j) the Jacobian, or
 * nothing when jac is NULL.  Host arrays; returns when the results are in. */
int  scfd_chem_rates(const scfd_chem* chem, int n, const double* states, double* dndt, double* jac);

/* ---- CEA equilibrium thermochemistry (NASA/core) ------------------------ */
/* Per-cell chemical equilibrium at given density, internal energy and
 * fuel/oxidizer mass fractions: `cea` of store/therm_lib/NASA/core/sub_chem.f90
 * (1320-1651), a Newton iteration on the element potentials pi_i and ln T with
 * a dense (ne+1) x (ne+1) pivoted LU (NASA/core/LU.f90), NASA-9 polynomials
 * (NASA/core/thermo.inp, 7 coefficients + 2 integration constants per
 * temperature section) and Wilke-mixed viscosity fits (NASA/core/trans.inp).
 * Units follow the reference: n in mol/kg, E in J/kg, MW in g/mol. */
#define SCFD_CEA_MAX_SPECIES   32
#define SCFD_CEA_MAX_ELEMENTS  6
#define SCFD_CEA_MAX_SECTIONS  6   /* thermo temperature sections (chem module: co(9,6,:)) */
#define SCFD_CEA_MAX_TSECTIONS 3   /* viscosity temperature sections (trans(4,3,:))      */

/* Tables of one species set, as set_therm_data / set_trans_data /
 * read_fo_composition read them (sub_chem.f90:70-305). */
typedef struct scfd_cea_data {
    int32_t abi_version;
    int32_t ns, ne, nt;    /* species, elements, species with a viscosity fit */
    int32_t nsec[SCFD_CEA_MAX_SPECIES];                            /* num_sctn */
    double  trange[SCFD_CEA_MAX_SPECIES][SCFD_CEA_MAX_SECTIONS][2];/* Trange(1:2,l,j) K */
    double  co[SCFD_CEA_MAX_SPECIES][SCFD_CEA_MAX_SECTIONS][9];    /* co(1:9,l,j) */
    double  mw[SCFD_CEA_MAX_SPECIES];                              /* g/mol */
    double  ac[SCFD_CEA_MAX_SPECIES][SCFD_CEA_MAX_ELEMENTS];       /* Ac(i,j): atoms of element i in species j */
    double  mwe[SCFD_CEA_MAX_ELEMENTS];                            /* element weights, MW.inp */
    int32_t ntsec[SCFD_CEA_MAX_SPECIES];                           /* num_sctn_trans */
    int32_t tr2th[SCFD_CEA_MAX_SPECIES];                           /* 0-based species of each fit */
    double  trange_t[SCFD_CEA_MAX_SPECIES][SCFD_CEA_MAX_TSECTIONS][2];
    double  trans[SCFD_CEA_MAX_SPECIES][SCFD_CEA_MAX_TSECTIONS][4];/* ln mu = A ln T + B/T + C/T^2 + D */
    double  pf, Tf, po, To;                                        /* fuel / oxidizer stream, Pa and K */
    double  nf[SCFD_CEA_MAX_SPECIES], no[SCFD_CEA_MAX_SPECIES];    /* stream mole ratios */
    int32_t init_hp;       /* stream states by cea_hp at the stream's p, h (initialize_cea('hp'));
                              0: by cea at its rho, e (initialize_cea('uv')) */
    int32_t reserved[7];
} scfd_cea_data;

/* The fuel and oxidizer states initialize_cea('uv') derives
 * (sub_chem.f90:1136-1230): element amounts b0 (mol/kg), element mass
 * fractions, the equilibrium state of each stream at its own density and
 * energy, and the initial value of every cell's saved composition n_save. */
typedef struct scfd_cea_stream {
    double rho, p, T, e, h, mw, kappa, mu;
    double b0[SCFD_CEA_MAX_ELEMENTS];
    double ye[SCFD_CEA_MAX_ELEMENTS];
    double n[SCFD_CEA_MAX_SPECIES];
} scfd_cea_stream;
typedef struct scfd_cea_info {
    scfd_cea_stream fuel, oxidizer;
    double of;        /* oxidizer/fuel mass ratio of the stream compositions */
    double n_init;    /* n_save initial value: sum(no + nf) / ns */
    int32_t iters_fuel, iters_oxidizer;
    int32_t reserved[6];
} scfd_cea_info;

typedef struct scfd_cea scfd_cea;

/* Parses nothing: builds the element lists and masks of initialize_cea and
 * solves the two stream states.  SCFD_E_ARG for counts out of range. */
int  scfd_cea_create(const scfd_cea_data* data, scfd_cea** out);
int  scfd_cea_destroy(scfd_cea* cea);
int  scfd_cea_info_get(const scfd_cea* cea, scfd_cea_info* info);
/* One `cea` call per cell on DEVICE arrays, component-major: Y[2][ncell]
 * (fuel, oxidizer mass fractions), n[ns][ncell], Yv[ns][ncell],
 * vhi[ns][ncell], DHi[2][ncell]; T and n are the reference's intent(inout)
 * guess / result.  Outputs other than T and n may be NULL; iters[ncell]
 * receives the Newton iterations (0 when the entry state already satisfies
 * the convergence test).  Enqueued on `stream` (cudaStream_t or NULL). */
int  scfd_cea_solve(scfd_cea* cea, int64_t ncell, const double* rho, const double* Y, const double* e,
                    double* T, double* n, double* mwave, double* kappa, double* mu, double* Yv,
                    double* vhi, double* DHi, int32_t* iters, void* stream);
/* cea_hp (sub_chem.f90:1652-1962): equilibrium at fixed pressure p[ncell] (Pa)
 * and enthalpy h[ncell] (J/kg); T is the guess / result.  Outputs as
 * scfd_cea_solve (no DHi; vhi = Ru 1e3 T / MW h/RT as the routine forms it).
 * The reference's retry after a singular matrix has no bound; here it counts
 * towards the 500-iteration limit. */
int  scfd_cea_solve_hp(scfd_cea* cea, int64_t ncell, const double* p, const double* Y, const double* h, double* T,
                       double* n, double* mwave, double* kappa, double* mu, double* Yv, double* vhi,
                       int32_t* iters, void* stream);
/* cea_tp (sub_chem.f90:1963-2248): equilibrium at fixed p and T; h[ncell]
 * (J/kg, may be NULL) receives the mixture enthalpy.  Retry bounded as hp. */
int  scfd_cea_solve_tp(scfd_cea* cea, int64_t ncell, const double* p, const double* Y, const double* T, double* n,
                       double* h, double* mwave, double* kappa, double* mu, double* Yv, double* vhi,
                       int32_t* iters, void* stream);
/* Synchronises the last solve's stream and returns, in counts[0..1], the
 * cells of the solves since the previous call that stopped at the
 * 500-iteration limit (the reference prints "not converted. at cea" and goes
 * on) and that met a singular matrix twice (SCFD_E_SINGULAR is returned). */
int  scfd_cea_status(scfd_cea* cea, int64_t* counts);

/* ---- no-allocation entry point ------------------------------------------ */
/* Capacity of the library's static scratch for scfd_rms_noalloc: partial sums
 * of 64 blocks for each of at most SCFD_MAX_PLANES planes. */
#define SCFD_NOALLOC_MAX_BLOCKS 4096

/* scfd_rms with no device allocation (no counterpart in the reference; it is
 * for callers that cannot call cudaMalloc, e.g. a solver whose device arrays
 * come from its own OpenACC / CUDA Fortran data regions or memory pool).
 * d_q and d_qp are DEVICE arrays in the layout of scfd_upload,
 * q(1:dimq,-1:nimax+2,-1:njmax+2,Nplane); *d_rms (device) receives the square
 * root of the sum, over the interior cells, of the squared change of the
 * energy component between qp and q, divided by the number of interior cells.
 * Enqueued on `stream` (a cudaStream_t, or NULL); the caller synchronises.  No
 * context is needed.  Scratch is a static device array of
 * SCFD_NOALLOC_MAX_BLOCKS doubles that every GPU loading the library keeps
 * until exit; its address is looked up on the first call on each device, so
 * make that first call before any stream capture, and do not reset the device
 * (cudaDeviceReset) between calls.  Calls that overlap on the GPU share the
 * scratch and race.  Returns SCFD_E_ARG for a bad descriptor or more than
 * SCFD_MAX_PLANES planes. */
int  scfd_rms_noalloc(const scfd_desc* desc, const double* d_q, const double* d_qp, double* d_rms,
                      void* stream);

#ifdef __cplusplus
}
#endif

#endif /* SCFD_B200_H */
