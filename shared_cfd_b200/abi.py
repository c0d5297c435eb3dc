"""ctypes mirror of include/scfd_b200.h.

The structures here must match the header field for field; test_abi.py checks
the sizes against the compiled library.
"""
import ctypes as C

ABI_VERSION = 1
MAX_PLANES = 64
MAX_SPECIES = 32
MAX_REACTIONS = 256
MAX_TRANS_SEC = 5
BC_MAXVAL = 2 * MAX_SPECIES + 8
INNER_LOG = 128

# status codes
OK, E_ARG, E_CUDA, E_TNEWTON, E_CHEM, E_OMEGA, E_RESRATE, E_NAN, E_SPIN, E_CONNECT, E_IO, E_STATE, \
    E_UNSUPPORTED, E_SINGULAR = range(14)
STATUS_NAMES = {
    0: "OK", 1: "E_ARG", 2: "E_CUDA", 3: "E_TNEWTON", 4: "E_CHEM", 5: "E_OMEGA", 6: "E_RESRATE",
    7: "E_NAN", 8: "E_SPIN", 9: "E_CONNECT", 10: "E_IO", 11: "E_STATE", 12: "E_UNSUPPORTED",
    13: "E_SINGULAR",
}

DIM_2D, DIM_Q2D = 0, 1
DT_GLOBAL, DT_LOCAL, DT_FIXED = 0, 1, 2
SCHEME_EULER, SCHEME_LUSGS, SCHEME_NR, SCHEME_PRECON, SCHEME_DUAL, SCHEME_PRECON_LUSGS = 0, 2, 3, 4, 5, 6
RECON_UPWIND, RECON_MUSCL = 0, 1
THERMO_IDEAL, THERMO_CHEMKIN_COLD, THERMO_CHEMKIN_REACTIVE = 0, 1, 2
MU_REFERENCE, MU_SUTHERLAND = 0, 1
PREC_FP64, PREC_MIXED = 0, 1

BC_EXTRAP, BC_FIXED, BC_OUTFLOW_P, BC_SLIP, BC_NOSLIP, BC_FIXED_PIN = range(6)
SIDE_ILO, SIDE_IHI, SIDE_JLO, SIDE_JHI = range(4)


class Desc(C.Structure):
    _fields_ = [
        ("abi_version", C.c_int32),
        ("nplane", C.c_int32),
        ("ni", C.c_int32 * MAX_PLANES),
        ("nj", C.c_int32 * MAX_PLANES),
        ("ny", C.c_int32),
        ("dim", C.c_int32),
        ("dt_mode", C.c_int32),
        ("scheme", C.c_int32),
        ("recon", C.c_int32),
        ("viscous", C.c_int32),
        ("thermo", C.c_int32),
        ("mu_model", C.c_int32),
        ("precision", C.c_int32),
        ("quirk_q1", C.c_int32),
        ("num_internal_loop", C.c_int32),
        ("il_write", C.c_int32),
        ("phi_mus", C.c_double), ("k_mus", C.c_double),
        ("kappa", C.c_double), ("rgas", C.c_double), ("nu_gas", C.c_double),
        ("suth_mu0", C.c_double), ("suth_t0", C.c_double), ("suth_s", C.c_double),
        ("prandtl", C.c_double), ("schmidt", C.c_double),
        ("cfl", C.c_double),
        ("dt_fixed", C.c_double),
        ("omega_max", C.c_double), ("omega_min", C.c_double), ("dq_max", C.c_double),
        ("res_rate_warn", C.c_double), ("res_rate_err", C.c_double),
        ("chem_max_substeps", C.c_int32),
        ("pad0", C.c_int32),
        ("cfl_tau", C.c_double),
        ("reserved", C.c_int32 * 12),
    ]


class BC(C.Structure):
    _fields_ = [
        ("plane", C.c_int32),
        ("side", C.c_int32),
        ("first", C.c_int32),
        ("last", C.c_int32),
        ("kind", C.c_int32),
        ("pad", C.c_int32),
        ("value", C.c_double * (BC_MAXVAL + 2)),
    ]


class Chem(C.Structure):
    _fields_ = [
        ("ns", C.c_int32), ("nr", C.c_int32), ("nt", C.c_int32), ("pad0", C.c_int32),
        ("coeff", ((C.c_double * 7) * 2) * MAX_SPECIES),
        ("tthre", (C.c_double * 3) * MAX_SPECIES),
        ("mws", C.c_double * MAX_SPECIES),
        ("rstate", (C.c_int32 * 2) * MAX_REACTIONS),
        ("indnu", ((C.c_int32 * 3) * 2) * MAX_REACTIONS),
        ("numnu", (C.c_int32 * 2) * MAX_REACTIONS),
        ("snu", C.c_int32 * MAX_REACTIONS),
        ("exist_m", C.c_int32 * MAX_REACTIONS),
        ("numm", C.c_int32 * MAX_REACTIONS),
        ("indm", (C.c_int32 * MAX_SPECIES) * MAX_REACTIONS),
        ("men", (C.c_double * MAX_SPECIES) * MAX_REACTIONS),
        ("abe", (C.c_double * 3) * MAX_REACTIONS),
        ("cabe", (C.c_double * 3) * MAX_REACTIONS),
        ("troe", (C.c_double * 4) * MAX_REACTIONS),
        ("tr2th", C.c_int32 * MAX_SPECIES),
        ("num_sctn_trans", C.c_int32 * MAX_SPECIES),
        ("trange_trans", ((C.c_double * 2) * MAX_TRANS_SEC) * MAX_SPECIES),
        ("trans", ((C.c_double * 4) * MAX_TRANS_SEC) * MAX_SPECIES),
        ("rtol", C.c_double), ("atol", C.c_double),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("dt_grbl", C.c_double),
        ("tt", C.c_double),
        ("res", C.c_double), ("res1", C.c_double),
        ("omega", C.c_double),
        ("status", C.c_int32),
        ("inner_iters", C.c_int32),
        ("chem_attempts", C.c_int64),
        ("chem_fallback_cells", C.c_int64),
        ("res_warn", C.c_int32),
        ("reserved", C.c_int32 * 7),
    ]


class AdjDesc(C.Structure):
    """scfd_adj_desc: the discrete adjoint run of scfd_adjoint_run."""
    _fields_ = [
        ("abi_version", C.c_int32),
        ("nsteps", C.c_int32),
        ("snapshots", C.c_int32),
        ("obj_bc", C.c_int32),
        ("win_first", C.c_int32),
        ("win_last", C.c_int32),
        ("param_bc", C.c_int32),
        ("forward_only", C.c_int32),
        ("reserved", C.c_int32 * 8),
    ]


MAX_RANKS = 64
DREQ_DONE, DREQ_REDUCE, DREQ_HALO = 0, 1, 2


class DReq(C.Structure):
    """scfd_dreq: what the caller must communicate before the next scfd_dstep."""
    _fields_ = [
        ("kind", C.c_int32),
        ("nsum", C.c_int32),
        ("nmin", C.c_int32),
        ("nranks", C.c_int32),
        ("seg", C.c_int64),
        ("buf", C.c_void_p),
    ]


REACTOR_QUEUE, REACTOR_PER_LAUNCH = 0, 1
REACTOR_IGNITED, REACTOR_FELL_BACK, REACTOR_FAILED = 1, 2, 4


class ReactorDesc(C.Structure):
    _fields_ = [
        ("abi_version", C.c_int32),
        ("n", C.c_int32),
        ("mode", C.c_int32),
        ("max_substeps", C.c_int32),
        ("t_end", C.c_double),
        ("dT_ign", C.c_double),
        ("dt_call", C.c_double),
        ("reserved", C.c_int32 * 6),
    ]


# CEA equilibrium tables (scfd_cea_data / scfd_cea_info)
CEA_MAX_SPECIES, CEA_MAX_ELEMENTS, CEA_MAX_SECTIONS, CEA_MAX_TSECTIONS = 32, 6, 6, 3


class CeaData(C.Structure):
    _fields_ = [
        ("abi_version", C.c_int32),
        ("ns", C.c_int32),
        ("ne", C.c_int32),
        ("nt", C.c_int32),
        ("nsec", C.c_int32 * CEA_MAX_SPECIES),
        ("trange", C.c_double * (CEA_MAX_SPECIES * CEA_MAX_SECTIONS * 2)),
        ("co", C.c_double * (CEA_MAX_SPECIES * CEA_MAX_SECTIONS * 9)),
        ("mw", C.c_double * CEA_MAX_SPECIES),
        ("ac", C.c_double * (CEA_MAX_SPECIES * CEA_MAX_ELEMENTS)),
        ("mwe", C.c_double * CEA_MAX_ELEMENTS),
        ("ntsec", C.c_int32 * CEA_MAX_SPECIES),
        ("tr2th", C.c_int32 * CEA_MAX_SPECIES),
        ("trange_t", C.c_double * (CEA_MAX_SPECIES * CEA_MAX_TSECTIONS * 2)),
        ("trans", C.c_double * (CEA_MAX_SPECIES * CEA_MAX_TSECTIONS * 4)),
        ("pf", C.c_double),
        ("Tf", C.c_double),
        ("po", C.c_double),
        ("To", C.c_double),
        ("nf", C.c_double * CEA_MAX_SPECIES),
        ("no", C.c_double * CEA_MAX_SPECIES),
        ("init_hp", C.c_int32),
        ("reserved", C.c_int32 * 7),
    ]


class CeaStream(C.Structure):
    _fields_ = [(k, C.c_double) for k in ("rho", "p", "T", "e", "h", "mw", "kappa", "mu")] + [
        ("b0", C.c_double * CEA_MAX_ELEMENTS),
        ("ye", C.c_double * CEA_MAX_ELEMENTS),
        ("n", C.c_double * CEA_MAX_SPECIES),
    ]


class CeaInfo(C.Structure):
    _fields_ = [
        ("fuel", CeaStream),
        ("oxidizer", CeaStream),
        ("of", C.c_double),
        ("n_init", C.c_double),
        ("iters_fuel", C.c_int32),
        ("iters_oxidizer", C.c_int32),
        ("reserved", C.c_int32 * 6),
    ]


# Exported entry points: name -> (restype, argtypes); the prefix (scfd_ for the
# CUDA library) is added by bind().
_P = C.c_void_p
_D = C.POINTER(C.c_double)
SIGNATURES = {
    "abi_version": (C.c_int, []),
    "create": (C.c_int, [C.POINTER(Desc), C.POINTER(_P)]),
    "destroy": (C.c_int, [_P]),
    "last_error": (C.c_int, [_P, C.c_char_p, C.c_int]),
    "set_geometry": (C.c_int, [_P, C.c_int, _D, _D]),
    "set_connectivity": (C.c_int, [_P, C.POINTER(C.c_int32), C.c_int]),
    "set_bc": (C.c_int, [_P, C.POINTER(BC), C.c_int]),
    "set_chem": (C.c_int, [_P, C.POINTER(Chem)]),
    "commit": (C.c_int, [_P]),
    "upload": (C.c_int, [_P, _D, _D, _D, C.c_double]),
    "prepare": (C.c_int, [_P, C.c_int]),
    "step": (C.c_int, [_P, C.c_int, C.POINTER(Stats)]),
    "run": (C.c_int, [_P, C.c_int, C.c_int, C.POINTER(Stats)]),
    "rms": (C.c_int, [_P, _D]),
    "inner_log": (C.c_int, [_P, _D, _D, C.c_int]),
    "download": (C.c_int, [_P, _D, _D, _D, _D]),
    "download_qp": (C.c_int, [_P, _D]),
    "write_restart": (C.c_int, [_P, C.c_char_p, C.c_int]),
    "read_restart": (C.c_int, [_P, C.c_char_p, C.POINTER(C.c_int), _D]),
    "write_geometry": (C.c_int, [_P, C.c_char_p]),
    "get_stream": (C.c_int, [_P, C.POINTER(_P)]),
    "launch_count": (C.c_int, [_P, C.POINTER(C.c_int64)]),
    "profile": (C.c_int, [_P, C.c_int]),
    "tuning": (C.c_int, [_P, C.c_char_p, C.c_int]),
    "kernel_stats": (C.c_int, [_P, C.c_int, _D, C.POINTER(C.c_int64), C.c_char_p, C.c_int]),
    "adjoint_run": (C.c_int, [_P, C.POINTER(AdjDesc), _D, _D, C.POINTER(C.c_int64)]),
    "set_bc_values": (C.c_int, [_P, C.c_int, _D]),
    "set_partition": (C.c_int, [_P, C.POINTER(C.c_int32), C.c_int, C.c_int]),
    "dstep": (C.c_int, [_P, C.c_int, C.POINTER(DReq), C.POINTER(Stats)]),
    "reactors_create": (C.c_int, [C.POINTER(Chem), C.c_int, C.POINTER(_P)]),
    "reactors_destroy": (C.c_int, [_P]),
    "reactors_upload": (C.c_int, [_P, C.c_int, _D, _D]),
    "reactors_launch": (C.c_int, [_P, C.POINTER(ReactorDesc)]),
    "reactors_download": (C.c_int, [_P, _D, _D, _D, C.POINTER(C.c_int64), C.POINTER(C.c_int32)]),
    "reactors_run": (C.c_int, [_P, C.POINTER(ReactorDesc), _D, _D, _D, _D, _D, C.POINTER(C.c_int64),
                               C.POINTER(C.c_int32)]),
    "reactors_stream": (_P, [_P]),
    "reactors_launch_count": (C.c_int, [_P, C.POINTER(C.c_int64)]),
    "chem_rates": (C.c_int, [C.POINTER(Chem), C.c_int, _D, _D, _D]),
    "cea_create": (C.c_int, [C.POINTER(CeaData), C.POINTER(_P)]),
    "cea_destroy": (C.c_int, [_P]),
    "cea_info_get": (C.c_int, [_P, C.POINTER(CeaInfo)]),
    "cea_solve": (C.c_int, [_P, C.c_int64, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "cea_solve_hp": (C.c_int, [_P, C.c_int64, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "cea_solve_tp": (C.c_int, [_P, C.c_int64, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "cea_status": (C.c_int, [_P, C.POINTER(C.c_int64)]),
}
K_THERMO, K_BC, K_DT, K_CHEM, K_RESIDUAL, K_SWEEP_FWD, K_SWEEP_BWD, K_UPDATE, K_COPY, K_OTHER, K_PACK, K_COUNT = \
    range(12)


class Bound:
    """The entry points of one library, looked up with a name prefix."""

    def __init__(self, lib, prefix):
        self.lib = lib
        self.prefix = prefix
        for name, (res, args) in SIGNATURES.items():
            f = getattr(lib, prefix + name)
            f.restype = res
            f.argtypes = args
            setattr(self, name, f)


def dptr(a):
    """double* of a C-contiguous float64 numpy array (or None)."""
    if a is None:
        return None
    return a.ctypes.data_as(_D)
