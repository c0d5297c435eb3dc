"""Shared helpers of the parity tests: run one case through a library and
compare conserved variables."""
import numpy as np

from shared_cfd_b200.solver import Solver


def run_case(case, lib, nsteps, step0=1, prepare=True):
    s = Solver(case, lib=lib)
    try:
        s.upload()
        if prepare:
            s.prepare(step0)
        st = s.run(step0, nsteps) if nsteps > 0 else None
        q, w, vhi, tt = s.download()
        return {"q": q, "w": w, "vhi": vhi, "tt": tt, "stats": st}
    finally:
        s.close()


def interior_stack(case, arr):
    """All interior cells of all planes, shape (ncells, K)."""
    return np.concatenate([case.interior(arr, p).reshape(-1, arr.shape[-1]) for p in range(len(case.planes))])


def rel_l2(case, a, b):
    """||a-b||_2 / ||b||_2 over the interior cells of all planes."""
    A = interior_stack(case, a)
    B = interior_stack(case, b)
    return float(np.linalg.norm(A - B) / np.linalg.norm(B))


def rel_l2_per_component(case, a, b):
    """Largest per-component relative L2 error.  Each conserved variable is
    normalised by the norm of its physical group: species densities by the
    total density, the two momentum components by the momentum magnitude,
    the energy by itself (a component that is zero in exact arithmetic, e.g.
    rho*v of a 1-D problem, then measures rounding against its group)."""
    A = interior_stack(case, a)
    B = interior_stack(case, b)
    nY = case.nY
    rho = np.linalg.norm(B[:, :nY].sum(axis=1))
    mom = np.linalg.norm(B[:, nY:nY + 2])
    ene = np.linalg.norm(B[:, nY + 2])
    errs = []
    for k in range(B.shape[1]):
        den = rho if k < nY else (mom if k < nY + 2 else ene)
        errs.append(np.linalg.norm(A[:, k] - B[:, k]) / den)
    return float(max(errs)), errs
