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


def rel_l2_per_component(case, a, b, floor_frac=1e-12):
    """Largest per-component relative L2 error; each component is normalised
    by max(||b_k||, floor_frac * ||b||) so that components that are zero
    everywhere do not divide by zero."""
    A = interior_stack(case, a)
    B = interior_stack(case, b)
    tot = np.linalg.norm(B)
    errs = []
    for k in range(B.shape[1]):
        den = max(np.linalg.norm(B[:, k]), floor_frac * tot)
        errs.append(np.linalg.norm(A[:, k] - B[:, k]) / den)
    return float(max(errs)), errs
