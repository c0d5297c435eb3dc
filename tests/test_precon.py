"""The preconditioned schemes of store/time_scheme/precon/2d (SCFD_SCHEME_PRECON:
the NR inner loop with low-Mach preconditioning, local time step) and
store/time_scheme/preconLU-SGS/2d (SCFD_SCHEME_PRECON_LUSGS) on the CPU
restatement: a low-Mach case (the forward step's state, M ~ 0.14) stays finite
with a falling inner residual; where the reference velocity reaches the sound
speed the preconditioner is the identity (phi = 0, phh = -0) and
preconLU-SGS gives plain LU-SGS's result to rounding; both libraries refuse
the combinations checkout_flow.py:154-177 forbids (no GPU)."""
import ctypes as C

import numpy as np
import pytest

from shared_cfd_b200 import abi, cases
from shared_cfd_b200.solver import Solver

from helpers import rel_l2, run_case


def precon_case(scheme, orientation=0, n=12, inner=12, seed=4, u=50.0):
    case = cases.forward_step(orientation, n=n, scheme=scheme, dt_mode=abi.DT_LOCAL, viscous=1)
    if u != 50.0:
        for p in range(2):
            q, w, vhi = cases.ideal_state(case, 1.0, u, 10.0, 1e5)
            cases.fill_all(case, p, q, w, vhi)
    case = cases.perturb(case, seed=seed)
    case.desc.num_internal_loop = inner
    case.desc.res_rate_err = 1e300
    case.desc.res_rate_warn = 1e300
    case.desc.cfl = 0.8
    return case


@pytest.mark.parametrize("orientation", [0, 2])
def test_precon_inner_loop_converges_at_low_mach(orc, orientation):
    case = precon_case(abi.SCHEME_PRECON, orientation, inner=40)
    case.desc.omega_max, case.desc.dq_max = 1.0, 1e3
    s = Solver(case, lib=orc)
    try:
        s.upload()
        s.prepare(1)
        for k in range(1, 4):
            st = s.step(k)
            assert st.res / st.res1 < 1e-3, (k, st.res / st.res1)
        q = s.download()[0]
        assert np.isfinite(q).all()
    finally:
        s.close()


def test_precon_lusgs_steps_stay_finite_and_damp_the_perturbation(orc):
    case = precon_case(abi.SCHEME_PRECON_LUSGS)
    a = run_case(case, orc, 5)
    b = run_case(case, orc, 60)
    assert np.isfinite(b["q"]).all()
    ref = run_case(case, orc, 0, prepare=True)
    # distance from the initial perturbed field grows, the solution stays bounded
    assert rel_l2(case, a["q"], ref["q"]) > 0
    assert rel_l2(case, b["q"], ref["q"]) < 1.0


def test_precon_lusgs_is_lusgs_where_the_flow_is_supersonic(orc):
    """u = 1000 m/s (M ~ 2.7): Ur = c, phi = 0, phh = -0, so the precon
    Jacobians, right-hand side, spectral radii and local dt are LU-SGS's."""
    a = run_case(precon_case(abi.SCHEME_PRECON_LUSGS, u=1000.0), orc, 10)
    case = precon_case(abi.SCHEME_LUSGS, u=1000.0)
    b = run_case(case, orc, 10)
    assert rel_l2(case, a["q"], b["q"]) < 1e-12


@pytest.mark.parametrize("lib_name", ["orc", "cuda"])
def test_unsupported_combinations_are_refused(orc, lib_name):
    from shared_cfd_b200 import build
    lib = orc if lib_name == "orc" else abi.Bound(C.CDLL(build.build()), "scfd_")
    for scheme in (abi.SCHEME_PRECON, abi.SCHEME_PRECON_LUSGS):
        for change in ("global_dt", "q2d"):
            case = precon_case(scheme)
            if change == "global_dt":
                case.desc.dt_mode = abi.DT_GLOBAL
            else:
                case.desc.dim = abi.DIM_Q2D
            ctx = C.c_void_p()
            assert lib.create(C.byref(case.desc), C.byref(ctx)) == abi.E_UNSUPPORTED, (scheme, change)


@pytest.mark.parametrize("scheme", [abi.SCHEME_PRECON, abi.SCHEME_PRECON_LUSGS])
def test_precon_sharded_equals_unsharded(orc, scheme):
    """Block sharding (scfd_dstep on two in-process ranks): the preconditioned
    local dt, alpha and right-hand side are per cell, so each rank's planes get
    the unsharded bits."""
    from shared_cfd_b200.sharded import ShardedSolver, lockstep
    case = precon_case(scheme, orientation=1, inner=6)
    ref = run_case(case, orc, 3)
    ranks = [ShardedSolver(case, [0, 1], lib=orc, rank=r, nranks=2) for r in range(2)]
    try:
        for s in ranks:
            s.upload()
            s.prepare(1)
        for n in range(3):
            lockstep(ranks, n + 1)
        for r, s in enumerate(ranks):
            q = s.download()[0]
            assert np.array_equal(case.interior(q, r), case.interior(ref["q"], r))
    finally:
        for s in ranks:
            s.close()
