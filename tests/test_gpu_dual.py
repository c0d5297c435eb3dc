"""The preconditioned dual time on the CUDA library (generic coefficient
sweep with the Gamma^-1 / S / S^-1 stages) against the CPU restatement:
FP64 within 1e-10 relative L2 of q, the mixed path within 1e-4, and the
sharded step bit-identical to the unsharded one."""
import numpy as np
import pytest

from shared_cfd_b200 import abi
from shared_cfd_b200.sharded import ShardedSolver, lockstep

from helpers import rel_l2, run_case
from test_dual import dual_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("orientation,viscous", [(0, 1), (2, 0), (3, 1)])
def test_dual_matches_restatement(gpu, orc, orientation, viscous):
    case = dual_case(orientation=orientation, n=24, viscous=viscous, inner=8)
    ref = run_case(case, orc, 5)
    got = run_case(case, gpu, 5)
    assert rel_l2(case, got["q"], ref["q"]) < 1e-10
    assert got["stats"].omega == pytest.approx(ref["stats"].omega, rel=1e-9)
    assert got["stats"].res == pytest.approx(ref["stats"].res, rel=1e-8)


def test_dual_mixed_precision(gpu, orc):
    case = dual_case(n=24, inner=8)
    ref = run_case(case, orc, 5)
    case.desc.precision = abi.PREC_MIXED
    got = run_case(case, gpu, 5)
    assert rel_l2(case, got["q"], ref["q"]) < 1e-4


def test_dual_sharded_equals_unsharded_gpu(gpu):
    case = dual_case(orientation=1, n=24, inner=6)
    ref = run_case(case, gpu, 3)
    ranks = [ShardedSolver(case, [0, 1], lib=gpu, rank=r, nranks=2) for r in range(2)]
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
