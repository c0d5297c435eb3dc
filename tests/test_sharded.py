"""Block-sharded steps (scfd_set_partition / scfd_dstep) on the CPU
restatement: ranks driven in lock step from one process and, through
torch.distributed, as two gloo processes.  A sharded run must give every plane
the bits of the unsharded run (the halo copies move values unchanged; dt and
omega are minima), the time and omega exactly, and the inner residual (a sum
over the ranks' planes, in another order) to rounding.  Also the argument and
state checks of both libraries (no GPU)."""
import ctypes as C
import os
import socket

import numpy as np
import pytest

from shared_cfd_b200 import abi, cases
from shared_cfd_b200.sharded import ShardedSolver, lockstep, partition_planes
from shared_cfd_b200.solver import Solver

from helpers import run_case


def _owned_planes_equal(case, ref, got, owner, rank, key="q"):
    for p in range(len(case.planes)):
        if owner[p] == rank:
            assert np.array_equal(case.interior(got[key], p), case.interior(ref[key], p)), (key, p)


def _lockstep_run(case, lib, owner, nranks, nsteps):
    ranks = [ShardedSolver(case, owner, lib=lib, rank=r, nranks=nranks) for r in range(nranks)]
    try:
        for s in ranks:
            s.upload()
            s.prepare(1)
        stats = None
        for n in range(nsteps):
            stats = lockstep(ranks, 1 + n)
        out = []
        for s in ranks:
            q, w, vhi, tt = s.download()
            out.append({"q": q, "w": w, "vhi": vhi, "tt": tt})
        return out, stats
    finally:
        for s in ranks:
            s.close()


def test_partition_balances_cells():
    assert partition_planes([512 * 512, 512 * 512, 512 * 256, 512 * 256], 2) == [0, 1, 0, 1]
    assert partition_planes([512 * 512, 512 * 512, 512 * 256, 512 * 256], 4) == [0, 1, 2, 3]
    assert partition_planes([10, 40, 30, 20], 2) == [0, 0, 1, 1]   # 50 cells each
    assert partition_planes([5, 5], 3) == [0, 1]


SCHEMES = [
    ("euler", abi.SCHEME_EULER, 0, abi.DIM_2D),
    ("lusgs", abi.SCHEME_LUSGS, 1, abi.DIM_2D),
    ("nr", abi.SCHEME_NR, 1, abi.DIM_Q2D),
]


@pytest.mark.parametrize("orientation", [0, 1, 2, 3])
@pytest.mark.parametrize("name,scheme,viscous,dim", SCHEMES)
def test_lockstep_two_ranks_match_unsharded(orc, orientation, name, scheme, viscous, dim):
    case = cases.perturb(cases.forward_step(orientation, n=8, scheme=scheme, viscous=viscous, dim=dim), seed=5)
    if scheme == abi.SCHEME_NR:
        case.desc.num_internal_loop = 4
        case.desc.res_rate_err = 1e300
    nsteps = 4
    ref = run_case(case, orc, nsteps)
    owner = [0, 1]
    got, stats = _lockstep_run(case, orc, owner, 2, nsteps)
    for r in range(2):
        for key in ("q", "w", "vhi"):
            _owned_planes_equal(case, ref, got[r], owner, r, key)
        assert got[r]["tt"] == ref["tt"]
        st = stats[r]
        assert st.status == 0
        assert st.dt_grbl == ref["stats"].dt_grbl
        assert st.omega == ref["stats"].omega
        assert st.inner_iters == ref["stats"].inner_iters
        assert st.res == pytest.approx(ref["stats"].res, rel=1e-12, abs=0.0)


def test_lockstep_reacting_step_four_and_three_ranks(orc):
    """The four-block reacting step (NR, chemistry, axisymmetric, viscous):
    one plane per rank, and three ranks with one holding two planes."""
    case = cases.reacting_step(scale=0.03, inner=3)
    ref = run_case(case, orc, 2)
    for owner in ([0, 1, 2, 3], [0, 1, 2, 2], [2, 0, 1, 0]):
        nr = max(owner) + 1
        got, stats = _lockstep_run(case, orc, owner, nr, 2)
        for r in range(nr):
            _owned_planes_equal(case, ref, got[r], owner, r, "q")
            _owned_planes_equal(case, ref, got[r], owner, r, "w")
            assert got[r]["tt"] == ref["tt"]
            assert stats[r].omega == ref["stats"].omega
        assert sum(s.chem_attempts for s in stats) == ref["stats"].chem_attempts


def test_lockstep_rank_without_planes(orc):
    case = cases.perturb(cases.forward_step(0, n=8, scheme=abi.SCHEME_LUSGS, viscous=1), seed=2)
    ref = run_case(case, orc, 3)
    owner = [0, 2]
    got, stats = _lockstep_run(case, orc, owner, 3, 3)
    for r in (0, 2):
        _owned_planes_equal(case, ref, got[r], owner, r, "q")
    assert stats[1].status == 0 and stats[1].dt_grbl == ref["stats"].dt_grbl


def test_sharded_rms_is_the_global_rms(orc):
    case = cases.perturb(cases.forward_step(1, n=8), seed=3)
    ranks = [ShardedSolver(case, [0, 1], lib=orc, rank=r, nranks=2) for r in range(2)]
    one = Solver(case, lib=orc)
    try:
        for s in ranks + [one]:
            s.upload()
        lockstep(ranks, 1)
        one.step(1)
        parts = [Solver.rms(s) for s in ranks]
        assert np.sqrt(sum(x * x for x in parts)) == pytest.approx(one.rms(), rel=1e-13)
        # the reference's combination (check_convergence.f90:17-33): each rank's
        # sqrt(sum) over its own cell count, summed over ranks
        ncell = case.ncells
        want = 0.0
        for s, part in zip(ranks, parts):
            want += part * ncell / s.owned_cells
        q, _, _, _ = one.download()
        qp = one.download_qp()
        direct = 0.0
        for p in range(len(case.planes)):
            d = case.interior(q, p)[:, :, case.D - 1] - case.interior(qp, p)[:, :, case.D - 1]
            direct += np.sqrt((d * d).sum()) / (case.ni[p] * case.nj[p])
        assert want == pytest.approx(direct, rel=1e-12)
    finally:
        for s in ranks + [one]:
            s.close()


def test_omega_floor_stops_every_rank(orc):
    """omega below omega_min on one rank's planes is every rank's E_OMEGA."""
    case = cases.perturb(cases.forward_step(0, n=8, scheme=abi.SCHEME_NR, viscous=1, dim=abi.DIM_Q2D), seed=5)
    case.desc.num_internal_loop = 3
    case.desc.omega_min = 1e30
    ref = Solver(case, lib=orc)
    try:
        ref.upload()
        assert ref.step(1, check=False).status == abi.E_OMEGA
    finally:
        ref.close()
    ranks = [ShardedSolver(case, [0, 1], lib=orc, rank=r, nranks=2) for r in range(2)]
    try:
        for s in ranks:
            s.upload()
        stats = lockstep(ranks, 1, check=False)
        assert [s.status for s in stats] == [abi.E_OMEGA, abi.E_OMEGA]
    finally:
        for s in ranks:
            s.close()


def _libs():
    from shared_cfd_b200 import build
    build.build()
    return [abi.Bound(C.CDLL(build.OUT), "scfd_")]


def test_partition_checks_without_gpu(orc):
    case = cases.forward_step(0, n=8)
    for lib in [orc] + _libs():
        ctx = C.c_void_p()
        assert lib.create(C.byref(case.desc), C.byref(ctx)) == 0
        try:
            own = (C.c_int32 * 2)(0, 2)
            assert lib.set_partition(ctx, own, 2, 0) == abi.E_ARG        # owner out of range
            own = (C.c_int32 * 2)(0, 1)
            assert lib.set_partition(ctx, own, 2, 2) == abi.E_ARG        # rank out of range
            assert lib.set_partition(ctx, own, 0, 0) == abi.E_ARG
            assert lib.set_partition(ctx, own, abi.MAX_RANKS + 1, 0) == abi.E_ARG
            assert lib.set_partition(ctx, own, 2, 1) == 0
            req, st = abi.DReq(), abi.Stats()
            req.kind = 7
            assert lib.dstep(ctx, 1, C.byref(req), C.byref(st)) == abi.E_STATE   # before commit
            assert req.kind == abi.DREQ_DONE
            assert lib.dstep(ctx, 1, None, C.byref(st)) == abi.E_ARG
        finally:
            lib.destroy(ctx)


def test_partitioned_context_refuses_plain_step(orc):
    case = cases.forward_step(0, n=8)
    s = ShardedSolver(case, [0, 1], lib=orc, rank=0, nranks=2)
    try:
        s.upload()
        assert s.lib.step(s.ctx, 1, C.byref(abi.Stats())) == abi.E_STATE
        assert s.lib.run(s.ctx, 1, 2, C.byref(abi.Stats())) == abi.E_STATE
    finally:
        s.close()


# ---------------------------------------------------------------------------
# two gloo processes
# ---------------------------------------------------------------------------
def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gloo_rank(rank, port, orc_path, out_dir):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=2, timeout=datetime.timedelta(seconds=60))
    try:
        lib = abi.Bound(C.CDLL(orc_path), "orc_")
        case = cases.reacting_step(scale=0.03, inner=3)
        owner = partition_planes([a * b for a, b in zip(case.ni, case.nj)], 2)
        s = ShardedSolver(case, owner, lib=lib)
        s.upload()
        s.prepare(1)
        st = s.run(1, 2)
        q, w, vhi, tt = s.gather()
        rms = s.rms()
        s.close()
        np.savez(os.path.join(out_dir, "rank%d.npz" % rank), q=q, w=w, tt=tt, res=st.res, omega=st.omega,
                 dt=st.dt_grbl, status=st.status, rms=rms, owner=np.array(owner))
    finally:
        dist.destroy_process_group()


def test_gloo_two_processes_match_unsharded(orc, tmp_path):
    import torch.multiprocessing as mp
    from conftest import ORACLE_SO
    port = _free_port()
    mp.start_processes(_gloo_rank, args=(port, ORACLE_SO, str(tmp_path)), nprocs=2, start_method="spawn")
    case = cases.reacting_step(scale=0.03, inner=3)
    ref = Solver(case, lib=orc)
    try:
        ref.upload()
        ref.prepare(1)
        st = ref.run(1, 2)
        q, w, vhi, tt = ref.download()
        rms = ref.rms()
    finally:
        ref.close()
    for r in range(2):
        got = np.load(os.path.join(tmp_path, "rank%d.npz" % r))
        for p in range(len(case.planes)):
            assert np.array_equal(case.interior(got["q"], p), case.interior(q, p)), p
            assert np.array_equal(case.interior(got["w"], p), case.interior(w, p)), p
        assert float(got["tt"]) == tt
        assert float(got["dt"]) == st.dt_grbl
        assert float(got["omega"]) == st.omega
        assert int(got["status"]) == 0
        assert float(got["res"]) == pytest.approx(st.res, rel=1e-12)
        assert float(got["rms"]) == pytest.approx(rms, rel=1e-12)


@pytest.mark.parametrize("orientation", [0, 1, 2, 3])
def test_split_planes_explicit_equals_unsplit(orc, orientation):
    """Cutting the blocks along i (the decomposition of multi-GPU runs) leaves
    an explicit inviscid step bit-identical: the two-layer halo copies give
    every face the neighbours it had in the whole block."""
    whole = cases.perturb(cases.forward_step(orientation, n=8), seed=4)
    cut = cases.split_planes_i(whole, 2)
    assert len(cut.planes) == 4
    r0 = run_case(whole, orc, 5)
    r2 = run_case(cut, orc, 5)
    for p in range(2):
        joined = np.concatenate([cut.interior(r2["q"], 2 * p), cut.interior(r2["q"], 2 * p + 1)], axis=1)
        assert np.array_equal(joined, whole.interior(r0["q"], p))
    assert r0["tt"] == r2["tt"]


def test_split_reacting_step_sharded_over_four_ranks(orc):
    """The decomposition bench.py uses on 4 GPUs: each block cut in two along
    i, one large and one small piece per rank."""
    case = cases.split_planes_i(cases.reacting_step(scale=0.0625, inner=3), 2)
    owner = partition_planes([a * b for a, b in zip(case.ni, case.nj)], 4)
    loads = [sum(a * b for a, b, o in zip(case.ni, case.nj, owner) if o == r) for r in range(4)]
    assert max(loads) == min(loads)
    ref = run_case(case, orc, 2)
    got, stats = _lockstep_run(case, orc, owner, 4, 2)
    for r in range(4):
        _owned_planes_equal(case, ref, got[r], owner, r, "q")
        assert stats[r].status == 0
