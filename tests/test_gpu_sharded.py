"""Block-sharded steps of the CUDA library on one GPU: the contexts of all ranks
live in this process and are driven in lock step (the requests are fulfilled
by device copies between their buffers, no process group), so the sharded
kernel sequence, the halo pack/unpack and the device halves of the reductions
run exactly as under NCCL.  Every owned plane must carry the bits of the
unsharded GPU run, the time and omega must be equal, the residual equal to
rounding."""
import numpy as np
import pytest

from shared_cfd_b200 import abi, cases
from shared_cfd_b200.sharded import ShardedSolver, lockstep
from shared_cfd_b200.solver import Solver

pytestmark = pytest.mark.gpu


def _unsharded(case, lib, nsteps):
    s = Solver(case, lib=lib)
    try:
        s.upload()
        s.prepare(1)
        st = s.run(1, nsteps)
        q, w, vhi, tt = s.download()
        return {"q": q, "w": w, "vhi": vhi, "tt": tt, "stats": st}
    finally:
        s.close()


def _sharded(case, lib, owner, nsteps):
    nr = max(owner) + 1
    ranks = [ShardedSolver(case, owner, lib=lib, rank=r, nranks=nr) for r in range(nr)]
    try:
        for s in ranks:
            s.upload()
            s.prepare(1)
        for n in range(nsteps):
            stats = lockstep(ranks, 1 + n)  # the last step's, as scfd_run reports
        outs = []
        for s in ranks:
            q, w, vhi, tt = s.download()
            outs.append({"q": q, "w": w, "vhi": vhi, "tt": tt})
        return outs, stats
    finally:
        for s in ranks:
            s.close()


def _check(case, ref, outs, stats, owner):
    for r, got in enumerate(outs):
        for p in range(len(case.planes)):
            if owner[p] != r:
                continue
            for key in ("q", "w", "vhi"):
                assert np.array_equal(case.interior(got[key], p), case.interior(ref[key], p)), (r, p, key)
        assert got["tt"] == ref["tt"]
        assert stats[r].status == ref["stats"].status
        assert stats[r].dt_grbl == ref["stats"].dt_grbl
        assert stats[r].omega == ref["stats"].omega
        assert stats[r].res == pytest.approx(ref["stats"].res, rel=1e-12, abs=0.0)


@pytest.mark.parametrize("precision", [abi.PREC_FP64, abi.PREC_MIXED])
@pytest.mark.parametrize("owner", [[0, 1, 0, 1], [0, 1, 2, 3], [1, 1, 1, 0]])
def test_reacting_step_sharded_equals_unsharded(gpu, owner, precision):
    case = cases.reacting_step(scale=0.125, inner=4, precision=precision)
    ref = _unsharded(case, gpu, 3)
    outs, stats = _sharded(case, gpu, owner, 3)
    _check(case, ref, outs, stats, owner)
    assert sum(s.chem_attempts for s in stats) == ref["stats"].chem_attempts


@pytest.mark.parametrize("orientation", [0, 2, 3])
@pytest.mark.parametrize("scheme,viscous,dim", [(abi.SCHEME_EULER, 0, abi.DIM_2D),
                                                (abi.SCHEME_LUSGS, 1, abi.DIM_2D),
                                                (abi.SCHEME_NR, 1, abi.DIM_Q2D)])
def test_forward_step_sharded_equals_unsharded(gpu, orientation, scheme, viscous, dim):
    case = cases.perturb(cases.forward_step(orientation, n=24, scheme=scheme, viscous=viscous, dim=dim), seed=5)
    if scheme == abi.SCHEME_NR:
        case.desc.num_internal_loop = 4
        case.desc.res_rate_err = 1e300
    ref = _unsharded(case, gpu, 4)
    outs, stats = _sharded(case, gpu, [0, 1], 4)
    _check(case, ref, outs, stats, [0, 1])


def test_legacy_sweeps_sharded(gpu, monkeypatch):
    monkeypatch.setenv("SCFD_SWEEP_LEGACY", "1")
    case = cases.reacting_step(scale=0.0625, inner=3)
    ref = _unsharded(case, gpu, 2)
    outs, stats = _sharded(case, gpu, [0, 1, 1, 0], 2)
    _check(case, ref, outs, stats, [0, 1, 1, 0])


def test_rank_without_planes(gpu):
    case = cases.perturb(cases.forward_step(0, n=24, scheme=abi.SCHEME_NR, viscous=1, dim=abi.DIM_Q2D), seed=5)
    case.desc.num_internal_loop = 3
    case.desc.res_rate_err = 1e300
    ref = _unsharded(case, gpu, 2)
    outs, stats = _sharded(case, gpu, [0, 2], 2)
    _check(case, ref, [outs[0], outs[1], outs[2]], stats, [0, 2])
