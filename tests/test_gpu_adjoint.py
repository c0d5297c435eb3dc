"""The discrete adjoint of the explicit ideal-gas step on the GPU
(scfd_adjoint_run): the objective equals the CPU restatement's, the gradient
with respect to the inflow values agrees with central finite differences of
the GPU objective to 1e-5, the checkpointing schedule changes the work but not
the gradient, and torch.autograd returns the same gradient."""
import numpy as np
import pytest

from shared_cfd_b200 import abi, cases
from shared_cfd_b200.adjoint import adjoint_run, boundary_objective, set_bc_values
from shared_cfd_b200.solver import Solver

pytestmark = pytest.mark.gpu

NSTEPS, WINDOW, OBJ, PARAM = 60, (10, 59), 2, 0


@pytest.fixture(scope="module")
def setup(gpu):
    case = cases.adjoint_channel(n=24)
    s = Solver(case, lib=gpu)
    s.upload()
    yield case, s
    s.close()


def test_objective_matches_restatement(setup, orc):
    case, s = setup
    J, _, _ = adjoint_run(s, NSTEPS, OBJ, WINDOW, forward_only=True)
    Jfull, _, _ = adjoint_run(s, NSTEPS, OBJ, WINDOW, PARAM, snapshots=4)
    assert Jfull == J
    o = Solver(case, lib=orc)
    try:
        o.upload()
        Jo, _, _ = adjoint_run(o, NSTEPS, OBJ, WINDOW, forward_only=True)
    finally:
        o.close()
    assert J == pytest.approx(Jo, rel=1e-12)


def test_gradient_matches_central_differences(setup):
    case, s = setup
    D = case.D
    J0, grad, counts = adjoint_run(s, NSTEPS, OBJ, WINDOW, PARAM, snapshots=8)
    base = np.array(case.bcs[PARAM].value[:])
    gmax = np.abs(grad[:case.W]).max()
    assert gmax > 0.0
    try:
        for k in (0, 1, 2, 3, D + 2):   # rho, u, v, p and h_t of the inflow ghost cells
            h = 1e-6 * max(abs(base[k]), 1.0)
            Jpm = []
            for sign in (1.0, -1.0):
                v = base.copy()
                v[k] += sign * h
                set_bc_values(s, PARAM, v)
                Jpm.append(adjoint_run(s, NSTEPS, OBJ, WINDOW, forward_only=True)[0])
            fd = (Jpm[0] - Jpm[1]) / (2 * h)
            assert abs(fd - grad[k]) <= 1e-5 * max(abs(grad[k]), 1e-3 * gmax), (k, fd, grad[k])
    finally:
        set_bc_values(s, PARAM, base)


def test_checkpointing_schedule_does_not_change_the_gradient(setup):
    case, s = setup
    out = {}
    for snaps in (0, 2, 8, 100):
        J, grad, counts = adjoint_run(s, NSTEPS, OBJ, WINDOW, PARAM, snapshots=snaps)
        out[snaps] = (J, grad, counts)
        assert counts[1] == NSTEPS
    assert out[100][2][0] == NSTEPS - 1                      # every state formed once
    assert out[0][2][0] == NSTEPS * (NSTEPS - 1) // 2         # no stored state: recompute from the start
    assert out[8][2][0] < 3 * NSTEPS
    for snaps in (0, 2, 8):
        assert out[snaps][0] == out[100][0]
        assert np.allclose(out[snaps][1], out[100][1], rtol=1e-12, atol=1e-12 * np.abs(out[100][1]).max())


def test_autograd_gives_the_adjoint_gradient(setup):
    import torch
    case, s = setup
    base = np.array(case.bcs[PARAM].value[:])
    _, grad, _ = adjoint_run(s, NSTEPS, OBJ, WINDOW, PARAM, snapshots=8)
    values = torch.tensor(base[:4], dtype=torch.float64, requires_grad=True)
    J = boundary_objective(values, s, PARAM, NSTEPS, OBJ, WINDOW, snapshots=8)
    J.backward()
    assert np.allclose(values.grad.numpy(), grad[:4], rtol=1e-12)
    set_bc_values(s, PARAM, base)
    s.upload()
