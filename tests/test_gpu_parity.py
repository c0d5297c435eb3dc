"""Parity of the CUDA path (called through the C ABI) with the CPU
restatement of the reference, on seeded inputs at sizes the restatement
finishes in seconds.

Tolerance for the plain (FP64) path: 1e-10 relative L2 of the conserved
variables after the stated step count.  Halo indexing is checked bit-exactly.
"""
import numpy as np
import pytest

from shared_cfd_b200 import abi, cases
from shared_cfd_b200.solver import Solver

from helpers import rel_l2, rel_l2_per_component, run_case

TOL_FP64 = 1e-10

pytestmark = pytest.mark.gpu


def _parity(case, gpu, orc, n, tol=TOL_FP64):
    a = run_case(case, gpu, n)
    b = run_case(case, orc, n)
    assert a["stats"] is None or a["stats"].status == 0
    assert np.isfinite(a["q"]).all()
    err = rel_l2(case, a["q"], b["q"])
    errk, _ = rel_l2_per_component(case, a["q"], b["q"])
    assert err <= tol, "rel L2 %g" % err
    assert errk <= 100 * tol, "per-component rel L2 %g" % errk
    return a, b, err


def test_sod_200_steps(gpu, orc):
    case = cases.sod()
    a, b, err = _parity(case, gpu, orc, 200)
    assert abs(a["tt"] - b["tt"]) <= 1e-12 * b["tt"]


@pytest.mark.parametrize("orientation", [0, 1, 2, 3])
def test_forward_step_euler_halo(gpu, orc, orientation):
    case = cases.perturb(cases.forward_step(orientation, n=10), seed=orientation)
    _parity(case, gpu, orc, 30)


@pytest.mark.parametrize("orientation", [0, 1, 2, 3])
def test_forward_step_lusgs_local_dt(gpu, orc, orientation):
    case = cases.perturb(cases.forward_step(orientation, n=10, scheme=abi.SCHEME_LUSGS, dt_mode=abi.DT_LOCAL,
                                            viscous=1), seed=10 + orientation)
    case.desc.cfl = 2.0
    _parity(case, gpu, orc, 10)


def test_flat_plate_lusgs(gpu, orc):
    case = cases.flat_plate(48, 40)
    _parity(case, gpu, orc, 20)


def test_nr_q2d_viscous_ideal(gpu, orc):
    case = cases.perturb(cases.forward_step(0, n=12, scheme=abi.SCHEME_NR, dt_mode=abi.DT_GLOBAL, viscous=1,
                                            dim=abi.DIM_Q2D), seed=7)
    case.desc.num_internal_loop = 6
    case.desc.res_rate_err = 1e300
    case.desc.omega_min = 0.0
    _parity(case, gpu, orc, 3)


def test_lusgs_wide_strips(gpu, orc):
    """More than one 32-row strip per plane and a partial last strip."""
    case = cases.perturb(cases.forward_step(1, n=37, scheme=abi.SCHEME_LUSGS, dt_mode=abi.DT_LOCAL), seed=3)
    case.desc.cfl = 3.0
    _parity(case, gpu, orc, 4)


def test_reacting_step_small(gpu, orc):
    case = cases.reacting_step(scale=1.0 / 32.0, inner=4)
    _parity(case, gpu, orc, 2)


def test_reacting_step_chemistry_goes_to_dvode(gpu, orc):
    """A premixed wake at 1500 K and dt = 1e-4 s: every wake cell's interval
    uses up its 10 CHEMEQ2 attempts, and k_chem_dvode finishes it with DVODE
    (sub_chem.f90:1755-1775) as the restatement does."""
    case = cases.reacting_step(scale=1.0 / 32.0, inner=4, dt=1e-4, wake="premixed")
    a = run_case(case, gpu, 2)
    b = run_case(case, orc, 2)
    sa, sb = a["stats"], b["stats"]
    assert sa.status == 0 and sb.status == 0
    wake = case.ni[3] * case.nj[3]
    assert sb.chem_fallback_cells >= wake
    assert sa.chem_fallback_cells == sb.chem_fallback_cells
    assert np.isfinite(a["q"]).all()
    err = rel_l2(case, a["q"], b["q"])
    assert err <= 1e-8, "rel L2 %g" % err


def test_halo_indexing_bit_exact(gpu, orc):
    """Ghost cells written by the halo copy and the boundary descriptors hold
    bit-identical values on both paths: q carries a unique density per cell
    and w(1) = q(1) exactly for the ideal gas."""
    for orientation in range(4):
        case = cases.forward_step(orientation, n=9)
        for p in range(2):
            nj, ni = case.nj[p], case.ni[p]
            jj, ii = np.meshgrid(np.arange(nj + 4), np.arange(ni + 4), indexing="ij")
            case.q[p, :nj + 4, :ni + 4, 0] = 1.0 + 1e-3 * (p * 10000 + jj * 100 + ii)
        a = run_case(case, gpu, 0)
        b = run_case(case, orc, 0)
        for p in range(2):
            nj, ni = case.nj[p], case.ni[p]
            ga = a["w"][p, :nj + 4, :ni + 4, 0]
            gb = b["w"][p, :nj + 4, :ni + 4, 0]
            assert np.array_equal(ga[1:-1, 1:-1], gb[1:-1, 1:-1]), "orientation %d plane %d" % (orientation, p)
            assert np.array_equal(ga[2:-2, 0], gb[2:-2, 0]) and np.array_equal(ga[0, 2:-2], gb[0, 2:-2])


def test_mixed_precision_error_is_stated(gpu, orc):
    """The FP32-reconstruction path stays close to the FP64 restatement."""
    case = cases.flat_plate(48, 40)
    b = run_case(case, orc, 20)
    case.desc.precision = abi.PREC_MIXED
    a = run_case(case, gpu, 20)
    err = rel_l2(case, a["q"], b["q"])
    assert err < 1e-4, err


def test_nan_is_reported(gpu):
    case = cases.sod(40, 4)
    case.q[0, 5, 10, 3] = np.nan
    s = Solver(case, lib=gpu)
    s.upload()
    s.prepare(1)
    s.run(1, 1, check=False)
    with pytest.raises(Exception):
        s.rms()
    s.close()


def test_launch_count_positive(gpu):
    case = cases.sod(40, 4)
    s = Solver(case, lib=gpu)
    s.upload()
    s.prepare(1)
    s.run(1, 3)
    assert s.launch_count() >= 3 * 4
    s.close()


SWEEP_ENV = {"lane": {}, "legacy": {"SCFD_SWEEP_LEGACY": "1"}}


@pytest.mark.parametrize("path", sorted(SWEEP_ENV))
def test_sweep_paths_agree(gpu, orc, path, monkeypatch):
    """Both sweep implementations match the restatement: strip records
    streamed by bulk copies (default) and the generic per-lane gather."""
    for k, val in SWEEP_ENV[path].items():
        monkeypatch.setenv(k, val)
    case = cases.perturb(cases.forward_step(2, n=20, scheme=abi.SCHEME_LUSGS, dt_mode=abi.DT_LOCAL, viscous=1,
                                            dim=abi.DIM_Q2D), seed=21)
    case.desc.cfl = 2.0
    _parity(case, gpu, orc, 5)


@pytest.mark.parametrize("path", sorted(SWEEP_ENV))
def test_sweep_many_tasks_ragged(gpu, orc, path, monkeypatch):
    """One plane of 150 rows: several strips, the last of them ragged, so the
    wavefront hands the top row of each strip to the next and ends in a
    partial strip."""
    for k, val in SWEEP_ENV[path].items():
        monkeypatch.setenv(k, val)
    case = cases.perturb(cases.flat_plate(40, 150), seed=5)
    _parity(case, gpu, orc, 3)


def test_reacting_step_two_tasks_per_plane(gpu, orc):
    """Reacting NR q2d step at a quarter of the resolution per direction:
    128- and 64-row planes, several strips per plane."""
    case = cases.reacting_step(scale=0.25, inner=3)
    _parity(case, gpu, orc, 1)


def test_graph_replay_matches_eager(gpu, monkeypatch):
    """Steps replayed from the captured CUDA graph give bit-identical states to
    the same kernels launched one by one."""
    out = {}
    for mode in ("eager", "graph"):
        if mode == "eager":
            monkeypatch.setenv("SCFD_GRAPH", "0")
        else:
            monkeypatch.delenv("SCFD_GRAPH", raising=False)
        case = cases.reacting_step(scale=1.0 / 32.0, inner=4, precision=abi.PREC_MIXED)
        s = Solver(case)
        s.upload()
        s.prepare(1)
        st = s.run(1, 4)
        assert st.status == 0
        out[mode] = (s.download()[0], s.launch_count())
        s.close()
    assert np.array_equal(out["eager"][0], out["graph"][0])
    assert out["eager"][1] == out["graph"][1]


@pytest.mark.parametrize("nj", [300, 520])
def test_sweep_tasks_hand_off_through_global_memory(gpu, orc, nj):
    """Planes of 10 and 17 strips: the wavefront runs as tasks of up to 8
    strips, so the top row of one task reaches the next through global memory
    (forward upwards, backward downwards), with a ragged last strip and a
    one-strip last task."""
    case = cases.perturb(cases.flat_plate(24, nj), seed=nj)
    _parity(case, gpu, orc, 3)
    case.desc.precision = abi.PREC_MIXED
    a = run_case(case, gpu, 3)
    assert a["stats"].status == 0 and np.isfinite(a["q"]).all()


def test_inner_log_matches_oracle(gpu, orc):
    """omega (from the Dqrate limiter) and the residual of every inner iteration
    of a reacting NR step agree with the restatement."""
    case = cases.reacting_step(scale=1.0 / 32.0, inner=5)
    logs = []
    for lib in (gpu, orc):
        s = Solver(case, lib=lib)
        try:
            s.upload()
            s.prepare(1)
            s.run(1, 2)
            logs.append(s.inner_log())
        finally:
            s.close()
    (om_g, res_g), (om_o, res_o) = logs
    assert len(om_g) == len(om_o) == 5
    np.testing.assert_allclose(om_g, om_o, rtol=1e-8)
    np.testing.assert_allclose(res_g, res_o, rtol=1e-8)


def test_reacting_step_full_size_one_step(gpu, orc):
    """The reacting-step workload at its full size (786 432 cells, 512-row
    planes run as two tasks each), one physical step of 20 inner iterations:
    FP64 within 1e-10 of the restatement."""
    case = cases.reacting_step(scale=1.0)
    _parity(case, gpu, orc, 1)


def _run_marks(case, lib, marks):
    s = Solver(case, lib=lib)
    try:
        s.upload()
        s.prepare(1)
        out, k = {}, 0
        for m in marks:
            st = s.run(k + 1, m - k)
            assert st.status == 0
            k = m
            out[m] = s.download()[0]
        return out
    finally:
        s.close()


def test_flat_plate_full_config(gpu, orc):
    """The flat-plate configuration as stated: 256x128 cells, LU-SGS with local
    time stepping, 5000 iterations.  The startup transient of this flow
    amplifies any rounding difference exponentially (measured FP64 GPU vs
    restatement: 1e-18 after 1 iteration, 3e-12 after 100, 1.5e-6 at the peak
    near iteration 500), and the difference then decays as both runs converge
    to the same steady state (9e-9 after 5000; the mixed path 1.3e-5).  So the
    FP64 path is held to 1e-10 after 100 iterations and to 5e-8 after 5000, and
    the mixed path's wall-normal profiles of u and T (at x = 0.05 m and 0.09 m)
    to 1e-4 of the restatement's after 5000."""
    case = cases.flat_plate(256, 128)
    marks = (100, 5000)
    a = _run_marks(case, gpu, marks)
    b = _run_marks(case, orc, marks)
    assert rel_l2(case, a[100], b[100]) <= TOL_FP64
    assert np.isfinite(a[5000]).all()
    assert rel_l2(case, a[5000], b[5000]) <= 5e-8
    case.desc.precision = abi.PREC_MIXED
    m = _run_marks(case, gpu, (5000,))[5000]
    D = case.D
    for x_frac in (0.5, 0.9):
        i = int(x_frac * case.ni[0])
        for name, f in (("u", lambda q: q[:, i, 1] / q[:, i, 0]),
                        ("T", lambda q: (q[:, i, D - 1] - 0.5 * (q[:, i, 1] ** 2 + q[:, i, 2] ** 2) / q[:, i, 0])
                         / q[:, i, 0])):
            pm = f(case.interior(m, 0))
            pb = f(case.interior(b[5000], 0))
            err = np.linalg.norm(pm - pb) / np.linalg.norm(pb)
            assert err <= 1e-4, "%s profile at x/L %.1f: %g" % (name, x_frac, err)


def test_reacting_step_runs_the_cluster_wavefront(gpu):
    """Both precisions of the reacting step take the cluster-wavefront sweep
    (not the generic fallback): 512-row planes in two tasks, 256-row in one."""
    for prec in (abi.PREC_FP64, abi.PREC_MIXED):
        s = Solver(cases.reacting_step(scale=1.0, precision=prec), lib=gpu)
        try:
            sw = s.tuning()["sweep"]
        finally:
            s.close()
        assert sw["kind"] == "cluster wavefront" and sw["tasks"] == 6 and sw["clusters"] >= 1, sw
