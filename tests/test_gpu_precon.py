"""The precon schemes (store/time_scheme/precon/2d, preconLU-SGS/2d) on the
GPU against the CPU restatement, through the C ABI, on the perturbed low-Mach
forward step (M ~ 0.14, where the preconditioner acts): FP64 within 1e-10
relative L2 of q.  The restatement forms the dense preconditioned Jacobians
(I + pre1 pre2^T) A as the reference does; the device applies them matrix-free."""
import numpy as np
import pytest

from shared_cfd_b200 import abi

from helpers import rel_l2, run_case
from test_precon import precon_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("orientation", [0, 1, 2, 3])
def test_precon_lusgs_matches_restatement(gpu, orc, orientation):
    case = precon_case(abi.SCHEME_PRECON_LUSGS, orientation)
    a = run_case(case, gpu, 20)
    b = run_case(case, orc, 20)
    assert np.isfinite(a["q"]).all()
    err = rel_l2(case, a["q"], b["q"])
    assert err <= 1e-10, err


@pytest.mark.parametrize("orientation", [0, 2])
def test_precon_matches_restatement(gpu, orc, orientation):
    case = precon_case(abi.SCHEME_PRECON, orientation, inner=12)
    a = run_case(case, gpu, 4)
    b = run_case(case, orc, 4)
    err = rel_l2(case, a["q"], b["q"])
    assert err <= 1e-10, err
    sa, sb = a["stats"], b["stats"]
    assert sa.res / sa.res1 == pytest.approx(sb.res / sb.res1, rel=1e-6)


def test_precon_mixed_precision_is_close(gpu, orc):
    case = precon_case(abi.SCHEME_PRECON, 0, inner=12)
    b = run_case(case, orc, 3)
    case.desc.precision = abi.PREC_MIXED
    a = run_case(case, gpu, 3)
    assert rel_l2(case, a["q"], b["q"]) <= 1e-4


@pytest.mark.parametrize("scheme", [abi.SCHEME_PRECON, abi.SCHEME_PRECON_LUSGS])
def test_precon_sharded_equals_unsharded_gpu(gpu, scheme):
    from shared_cfd_b200.sharded import ShardedSolver, lockstep
    case = precon_case(scheme, orientation=1, inner=6)
    ref = run_case(case, gpu, 3)
    ranks = [ShardedSolver(case, [0, 1], lib=gpu, rank=r, nranks=2) for r in range(2)]
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
