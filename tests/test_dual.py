"""The preconditioned dual time (SCFD_SCHEME_DUAL, store/time_scheme/dual/2d)
on the CPU restatement: it iterates the same BDF2 physical step as NR, so with
both inner loops converged the two agree to rounding; its inner residual
falls; its sharded step gives the unsharded bits; and both libraries refuse
the combinations checkout_flow.py:159-168 forbids (no GPU)."""
import ctypes as C

import numpy as np
import pytest

from shared_cfd_b200 import abi, cases
from shared_cfd_b200.sharded import ShardedSolver, lockstep
from shared_cfd_b200.solver import Solver

from helpers import rel_l2, run_case


def dual_case(orientation=0, n=12, viscous=1, inner=30, cfl_tau=5.0, seed=3):
    case = cases.perturb(cases.forward_step(orientation, n=n, scheme=abi.SCHEME_DUAL, viscous=viscous), seed=seed)
    case.desc.num_internal_loop = inner
    case.desc.cfl_tau = cfl_tau
    case.desc.res_rate_err = 1e300
    return case


def test_dual_and_nr_converge_to_the_same_bdf2_step(orc):
    out = {}
    for scheme in (abi.SCHEME_NR, abi.SCHEME_DUAL):
        case = dual_case(inner=400)
        case.desc.scheme = scheme
        case.desc.omega_max, case.desc.dq_max = 1.0, 1e3
        s = Solver(case, lib=orc)
        try:
            s.upload()
            s.prepare(1)
            st = s.step(1)
            assert st.res / st.res1 < 1e-20
            out[scheme] = s.download()[0]
        finally:
            s.close()
    assert rel_l2(case, out[abi.SCHEME_DUAL], out[abi.SCHEME_NR]) < 1e-13


@pytest.mark.parametrize("viscous", [0, 1])
def test_dual_inner_residual_falls(orc, viscous):
    case = dual_case(viscous=viscous)
    s = Solver(case, lib=orc)
    try:
        s.upload()
        s.prepare(1)
        for n in range(3):
            st = s.step(n + 1)
            assert st.status == 0 and st.inner_iters == case.desc.num_internal_loop - 1
            assert st.res / st.res1 < 0.2
        assert np.isfinite(s.download()[0]).all()
    finally:
        s.close()


def test_dual_sharded_equals_unsharded(orc):
    case = dual_case(orientation=1, inner=6)
    ref = run_case(case, orc, 3)
    ranks = [ShardedSolver(case, [0, 1], lib=orc, rank=r, nranks=2) for r in range(2)]
    try:
        for s in ranks:
            s.upload()
            s.prepare(1)
        for n in range(3):
            stats = lockstep(ranks, n + 1)
        for r, s in enumerate(ranks):
            q = s.download()[0]
            assert np.array_equal(case.interior(q, r), case.interior(ref["q"], r))
            assert stats[r].omega == ref["stats"].omega
    finally:
        for s in ranks:
            s.close()


def test_dual_forbidden_combinations_without_gpu(orc):
    from shared_cfd_b200 import build
    build.build()
    libs = [orc, abi.Bound(C.CDLL(build.OUT), "scfd_")]
    for lib in libs:
        for change, code in ((("dim", abi.DIM_Q2D), abi.E_UNSUPPORTED), (("dt_mode", abi.DT_LOCAL), abi.E_UNSUPPORTED),
                             (("thermo", abi.THERMO_CHEMKIN_REACTIVE), abi.E_UNSUPPORTED),
                             (("cfl_tau", 0.0), abi.E_ARG)):
            case = dual_case()
            setattr(case.desc, change[0], change[1])
            ctx = C.c_void_p()
            assert lib.create(C.byref(case.desc), C.byref(ctx)) == code, change
        ctx = C.c_void_p()
        assert lib.create(C.byref(dual_case().desc), C.byref(ctx)) == 0
        lib.destroy(ctx)
