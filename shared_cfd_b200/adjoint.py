"""Gradients through the explicit ideal-gas step: the host side of
scfd_adjoint_run (include/scfd_b200.h).

The objective is the pressure force on one boundary, summed over a window of
steps; the parameters are the values of one boundary descriptor (the state of
a fixed inflow).  `adjoint_run` calls the library's reverse sweep (binomial
checkpointing of the states on the device); `BoundaryObjective` puts it behind
torch.autograd so that an inflow state held in a tensor gets its gradient by
`backward()`.
"""
import ctypes as C

import numpy as np

from . import abi


def adjoint_run(solver, nsteps, obj_bc, window=None, param_bc=-1, snapshots=16, forward_only=False):
    """Runs nsteps from the solver's uploaded state; returns (J, grad, counts).
    window: (first, last) steps whose states enter J (default: all).  grad has
    one entry per value[] of descriptor param_bc (zeros if param_bc < 0);
    counts = (forward steps, reverse steps)."""
    d = abi.AdjDesc()
    d.abi_version = abi.ABI_VERSION
    d.nsteps = nsteps
    d.snapshots = snapshots
    d.obj_bc = obj_bc
    first, last = window if window is not None else (0, nsteps - 1)
    d.win_first, d.win_last = first, last
    d.param_bc = param_bc
    d.forward_only = 1 if forward_only else 0
    J = C.c_double()
    grad = np.zeros(abi.BC_MAXVAL + 2)
    counts = (C.c_int64 * 2)()
    solver._check(solver.lib.adjoint_run(solver.ctx, C.byref(d), C.byref(J), abi.dptr(grad), counts), "adjoint_run")
    return J.value, grad, (counts[0], counts[1])


def set_bc_values(solver, bc, values):
    """Replaces value[] of descriptor bc (0-based) after commit."""
    v = np.zeros(abi.BC_MAXVAL + 2)
    v[:] = np.asarray(solver.case.bcs[bc].value[:], dtype=np.float64)
    v[:len(values)] = values
    solver._check(solver.lib.set_bc_values(solver.ctx, bc, abi.dptr(v)), "set_bc_values")
    for k in range(len(values)):
        solver.case.bcs[bc].value[k] = float(values[k])


def _function():
    import torch

    class BoundaryObjective(torch.autograd.Function):
        """J(values): values (1-d float64 tensor) replace the first entries of
        descriptor param_bc's value[]; the run starts from the case's initial
        state each time."""

        @staticmethod
        def forward(ctx, values, solver, param_bc, nsteps, obj_bc, window, snapshots):
            set_bc_values(solver, param_bc, values.detach().cpu().numpy())
            solver.upload()
            J, grad, _ = adjoint_run(solver, nsteps, obj_bc, window, param_bc, snapshots)
            ctx.save_for_backward(torch.as_tensor(grad[:values.numel()], dtype=values.dtype))
            return torch.tensor(J, dtype=values.dtype)

        @staticmethod
        def backward(ctx, gJ):
            (g,) = ctx.saved_tensors
            return gJ * g, None, None, None, None, None, None

    return BoundaryObjective


def boundary_objective(values, solver, param_bc, nsteps, obj_bc, window=None, snapshots=16):
    """torch-differentiable J of the inflow values (see BoundaryObjective)."""
    return _function().apply(values, solver, param_bc, nsteps, obj_bc, window, snapshots)
