"""The discrete adjoint of the explicit ideal-gas step, CPU side: the reverse
of the MUSCL face states, the SLAU flux and the primitive map
(shared_cfd_b200/csrc/adj_face.cuh) against central differences of the
forward functions, and the objective of scfd_adjoint_run on the CPU
restatement against the same sum formed from the states it steps through."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from shared_cfd_b200 import abi, cases
from shared_cfd_b200.adjoint import adjoint_run
from shared_cfd_b200.solver import Solver, SolverError

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "shared_cfd_b200", "csrc")


def test_reverse_functions_match_central_differences(tmp_path):
    exe = str(tmp_path / "face_check")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-I", CSRC, os.path.join(HERE, "adj", "face_check.cpp"),
                           "-o", exe])
    out = subprocess.check_output([exe], text=True)
    worst = {ln.split()[0]: float(ln.split()[1]) for ln in out.strip().splitlines()}
    assert set(worst) == {"muscl", "slau", "prim", "pressure"}
    for name, err in worst.items():
        assert err < 1e-7, (name, err)


def _pressure_force(case, q, bc):
    """sum over the descriptor's first interior cells of ds * p, from q."""
    b = case.bcs[bc]
    p = b.plane - 1
    xh, rh = case.planes[p]
    ni, nj = case.ni[p], case.nj[p]
    kap = case.desc.kappa
    tot = 0.0
    for s in range(b.first, b.last + 1):
        if b.side == abi.SIDE_JLO:
            i, j = s, 1
            ds = np.hypot(xh[s, 0] - xh[s - 1, 0], rh[s, 0] - rh[s - 1, 0])
        elif b.side == abi.SIDE_ILO:
            i, j = 1, s
            ds = np.hypot(xh[0, s] - xh[0, s - 1], rh[0, s] - rh[0, s - 1])
        else:
            raise NotImplementedError
        c = q[p, j + 1, i + 1]
        rho = c[:case.nY].sum()
        tot += ds * (kap - 1.0) * (c[case.nY + 2] - 0.5 * (c[case.nY] ** 2 + c[case.nY + 1] ** 2) / rho)
    return tot


@pytest.mark.parametrize("obj_bc", [2, 4])
def test_restatement_objective_is_the_window_sum(orc, obj_bc):
    case = cases.adjoint_channel(n=12)
    s = Solver(case, lib=orc)
    try:
        s.upload()
        J, _, counts = adjoint_run(s, 20, obj_bc, (4, 15), forward_only=True)
        assert counts == (15, 0)
        s.upload()
        ref = 0.0
        for n in range(16):
            if n >= 4:
                ref += _pressure_force(case, s.download()[0], obj_bc)
            if n < 15:
                s.step(n + 1)
        assert J == pytest.approx(ref, rel=1e-12)
    finally:
        s.close()


def test_restatement_has_no_reverse_and_checks_its_arguments(orc):
    case = cases.adjoint_channel(n=12)
    s = Solver(case, lib=orc)
    try:
        s.upload()
        with pytest.raises(SolverError) as e:
            adjoint_run(s, 10, 2, (0, 9), param_bc=0)
        assert e.value.code == abi.E_UNSUPPORTED
        with pytest.raises(SolverError) as e:
            adjoint_run(s, 10, 2, (3, 10), forward_only=True)
        assert e.value.code == abi.E_ARG
        with pytest.raises(SolverError) as e:
            adjoint_run(s, 10, 9, (0, 9), forward_only=True)
        assert e.value.code == abi.E_ARG
    finally:
        s.close()
