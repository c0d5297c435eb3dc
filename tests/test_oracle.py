"""Properties of the CPU restatement itself (it is the checker of the CUDA
path, so it is pinned here by properties the reference method has)."""
import numpy as np

from shared_cfd_b200 import abi, cases
from shared_cfd_b200.solver import Case

from helpers import interior_stack, run_case


def test_sod_conserves_mass_and_moves_the_shock(orc):
    case = cases.sod()
    r = run_case(case, orc, 200)
    q = case.interior(r["q"], 0)
    q0 = case.interior(case.q, 0)
    assert abs(q[:, :, 0].sum() / q0[:, :, 0].sum() - 1.0) < 1e-13
    assert abs(q[:, :, 3].sum() / q0[:, :, 3].sum() - 1.0) < 1e-13
    rho = q[1, :, 0]
    # contact + shock to the right of x = 0.5, rarefaction to the left
    assert rho[int(0.45 * 400)] < 1.0 and rho[int(0.55 * 400)] > 0.125
    assert np.all(np.diff(rho[:200]) <= 1e-12)   # monotone rarefaction


def _split_case(case2, scheme):
    """One block equal to the two blocks of forward_step orientation 0."""
    xh1, rh1 = case2.planes[0]
    xh2, rh2 = case2.planes[1]
    xh = np.concatenate([xh1, xh2[1:]], axis=0)
    rh = np.concatenate([rh1, rh2[1:]], axis=0)
    d = cases.base_desc(scheme=scheme, cfl=case2.desc.cfl)
    one = Case([(xh, rh)], d, bcs=cases.all_sides([(xh.shape[0] - 1, xh.shape[1] - 1)], abi.BC_EXTRAP))
    n1 = case2.ni[0]
    for arr1, arr2, dst in ((case2.q[0], case2.q[1], one.q), (case2.w[0], case2.w[1], one.w),
                            (case2.vhi[0], case2.vhi[1], one.vhi)):
        dst[0, :, :n1 + 2] = arr1[:, :n1 + 2]
        dst[0, :, n1 + 2:] = arr2[:, 2:dst.shape[2] - n1]
    return one


def test_halo_split_equals_single_block_explicit(orc):
    """Euler explicit: two blocks joined by the halo copy give bit-identical
    results to one block over the same cells."""
    two = cases.forward_step(0, n=8)
    two.bcs = [b for b in two.bcs]
    one = _split_case(two, abi.SCHEME_EULER)
    r2 = run_case(two, orc, 10)
    r1 = run_case(one, orc, 10)
    n1 = two.ni[0]
    a = np.concatenate([two.interior(r2["q"], 0), two.interior(r2["q"], 1)], axis=1)
    b = one.interior(r1["q"], 0)
    assert np.array_equal(a, b)


def test_axisymmetric_uniform_flow_is_preserved(orc):
    """q2d: the pressure source Area*p balances the r-weighted pressure flux of
    a uniform axial flow, inviscid and viscous."""
    for visc in (0, 1):
        case = cases.forward_step(1, n=8, viscous=visc, dim=abi.DIM_Q2D)
        for p in range(2):
            q, w, vhi = cases.ideal_state(case, 1.2, 100.0, 0.0, 1e5)
            cases.fill_all(case, p, q, w, vhi)
        r = run_case(case, orc, 5)
        A = interior_stack(case, r["q"])
        B = interior_stack(case, case.q)
        assert np.abs(A - B).max() / np.abs(B).max() < 1e-12


def test_nr_inner_loop_runs_n_minus_1_iterations(orc):
    case = cases.forward_step(0, n=6, scheme=abi.SCHEME_NR, dt_mode=abi.DT_GLOBAL)
    case.desc.num_internal_loop = 4
    case.desc.res_rate_err = 1e300
    r = run_case(case, orc, 1)
    assert r["stats"].inner_iters == 3


def test_omega_floor_is_reported(orc):
    case = cases.perturb(cases.reacting_step(scale=1.0 / 64.0, inner=2), seed=1)
    case.desc.omega_min = 0.5
    case.desc.dq_max = 1e-9   # positivity limiter: omega = min(-q/Dq) * Dqmax
    from shared_cfd_b200.solver import Solver
    s = Solver(case, lib=orc)
    s.upload()
    s.prepare(1)
    st = s.step(1, check=False)
    s.close()
    assert st.status == abi.E_OMEGA


def test_inner_log_records_every_inner_iteration(orc):
    """The internal_res.dat record (time_NR_viscous.f90:87-95): one omega and
    residual per inner iteration; the first residual is res1, the last is res,
    and the applied omega is the last candidate capped at omega_max."""
    from shared_cfd_b200.solver import Solver
    case = cases.reacting_step(scale=1.0 / 64.0, inner=4)
    s = Solver(case, lib=orc)
    try:
        s.upload()
        s.prepare(1)
        st = s.step(1)
        om, res = s.inner_log()
    finally:
        s.close()
    assert len(om) == len(res) == 4
    assert res[0] == st.res1 and res[-1] == st.res
    assert min(case.desc.omega_max, om[-1]) == st.omega
    assert np.all(om > 0.0) and np.all(res > 0.0)
