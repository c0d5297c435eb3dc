"""Block-sharded runs: one process per GPU, each updating the planes it owns.

The host side of scfd_set_partition / scfd_dstep (include/scfd_b200.h).  It
takes the place of the reference's MPI layer: the cross-rank halo copies of
set_BC (MPI_Isend/Recv of w and vhi, store/cond/no-nV/condition.tail.f90:
71-330), the MPI_Allreduce MIN of dt_grbl (store/time_step/global/
set_dt.f90:40), the MPI_Reduce of omega and of the inner residual
(store/time_scheme/NR/q2d/time_NR_viscous.f90:87-90; here every rank receives
them) and of the RMS (store/core/check_convergence.f90:33).  The collectives
are torch.distributed's: NCCL between GPUs, gloo between CPU processes.

The library returns, at each point of a physical step where the ranks must
agree, a request; `ShardedSolver.dstep` fulfils it and continues.  The
exchange buffers of the CUDA library are device memory on the context's
stream: the collectives run with that stream current, so they are ordered
after the kernels that filled the buffer and before those that read it, with
no host synchronisation.  `lockstep` drives the contexts of all ranks from a
single process instead (no process group), e.g. to check the sharded kernels
on one GPU.
"""
import contextlib
import ctypes as C

import numpy as np

from . import abi
from .solver import Solver


def partition_planes(cells, nranks):
    """owner[p] for planes of `cells[p]` cells: planes in decreasing size, each
    to the rank with the fewest cells so far (lowest rank on ties)."""
    load = [0] * nranks
    owner = [0] * len(cells)
    for p in sorted(range(len(cells)), key=lambda k: (-cells[k], k)):
        r = min(range(nranks), key=lambda k: (load[k], k))
        owner[p] = r
        load[r] += cells[p]
    return owner


class _CudaBuf:
    """A device array of doubles owned by the library, for torch.as_tensor."""

    def __init__(self, addr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (addr, False), "version": 2}


class ShardedSolver(Solver):
    """One rank of a block-sharded run.

    owner:  owner[p], the rank of plane p (e.g. partition_planes)
    group:  torch.distributed process group (None: the default group), or
            None together with rank/nranks given for `lockstep` use
    """

    def __init__(self, case, owner, lib=None, group=None, rank=None, nranks=None):
        if rank is None or nranks is None:
            import torch.distributed as dist
            rank = dist.get_rank(group)
            nranks = dist.get_world_size(group)
        self.rank, self.nranks, self.group = rank, nranks, group
        self.owner = list(owner)
        super().__init__(case, lib=lib, partition=(self.owner, nranks, rank))
        self._device = self.stream() is not None
        self._views = {}
        self._run_launches = 0

    @property
    def owned_cells(self):
        return sum(a * b for a, b, o in zip(self.case.ni, self.case.nj, self.owner) if o == self.rank)

    # -- request buffers ---------------------------------------------------
    def buffer(self, addr, n):
        """torch view (no copy) of n doubles at the library address addr."""
        import torch
        key = (addr, n)
        t = self._views.get(key)
        if t is None:
            if self._device:
                t = torch.as_tensor(_CudaBuf(addr, n), device="cuda")
            else:
                t = torch.from_numpy(np.ctypeslib.as_array(C.cast(addr, C.POINTER(C.c_double)), shape=(n,)))
            self._views[key] = t
        return t

    def on_stream(self):
        """Makes the context's stream current for torch (a no-op on the CPU)."""
        if not self._device:
            return contextlib.nullcontext()
        import torch
        return torch.cuda.stream(torch.cuda.ExternalStream(self.stream()))

    def fulfil(self, req):
        import torch.distributed as dist
        if req.kind == abi.DREQ_REDUCE:
            t = self.buffer(req.buf, req.nsum + req.nmin)
            with self.on_stream():
                if req.nsum:
                    dist.all_reduce(t[:req.nsum], op=dist.ReduceOp.SUM, group=self.group)
                if req.nmin:
                    dist.all_reduce(t[req.nsum:], op=dist.ReduceOp.MIN, group=self.group)
        elif req.kind == abi.DREQ_HALO:
            seg = req.seg
            if seg == 0:
                return
            t = self.buffer(req.buf, seg * req.nranks)
            with self.on_stream():
                mine = t[self.rank * seg:(self.rank + 1) * seg].clone()
                dist.all_gather_into_tensor(t, mine, group=self.group)
        else:
            raise RuntimeError("unknown request %d" % req.kind)

    # -- stepping ----------------------------------------------------------
    def dstep(self, step=1, check=True):
        req, st = abi.DReq(), abi.Stats()
        while True:
            code = self.lib.dstep(self.ctx, step, C.byref(req), C.byref(st))
            if req.kind == abi.DREQ_DONE:
                break
            self.fulfil(req)
        if check:
            self._check(code, "dstep")
        return st

    def step(self, step=1, check=True):
        return self.dstep(step, check)

    def run(self, step, nsteps, check=True):
        st = None
        self._run_launches = 0
        for n in range(nsteps):
            st = self.dstep(step + n, check)
            self._run_launches += Solver.launch_count(self)
            if st.status:
                break
        return st

    def launch_count(self):
        """Kernels launched by the last run() (scfd_launch_count covers one step)."""
        return self._run_launches

    def rms(self, combine="global"):
        """The convergence RMS of the sharded case.

        The library returns this rank's share sqrt(tmp_r) / N, with tmp_r the
        rank's sum of squared energy changes and N the cells of the whole case.

        combine="global" (default): sqrt(sum_r tmp_r) / N, the value of the same
        case run unsharded on one GPU, independent of the rank count.

        combine="reference": sum_r sqrt(tmp_r) / n_r with n_r the rank's own
        cells, what check_convergence.f90:17-33 MPI_Reduce-sums over the
        reference's ranks.  With R equal ranks it is R**1.5 times the global
        value, so a min_RMS threshold taken from an R-rank run of the reference
        corresponds to min_RMS / R**1.5 in the global form."""
        import torch
        import torch.distributed as dist
        local = Solver.rms(self)
        dev = "cuda" if self._device else "cpu"
        if combine == "reference":
            own = self.owned_cells
            part = local * self.case.ncells / own if own else 0.0
            t = torch.tensor([part], dtype=torch.float64, device=dev)
            dist.all_reduce(t, group=self.group)
            return float(t.item())
        if combine != "global":
            raise ValueError("combine must be 'global' or 'reference'")
        t = torch.tensor([local * local], dtype=torch.float64, device=dev)
        dist.all_reduce(t, group=self.group)
        return float(np.sqrt(t.item()))

    def gather(self):
        """(q, w, vhi, tt) of the whole case on every rank, each plane (ghost
        layers included) from its owner."""
        import torch
        import torch.distributed as dist
        q, w, vhi, tt = self.download()
        mask = np.array([o == self.rank for o in self.owner])[:, None, None, None]
        dev = "cuda" if self._device else "cpu"
        out = []
        for a in (q, w, vhi):
            t = torch.from_numpy(np.where(mask, a, 0.0)).to(dev)
            dist.all_reduce(t, group=self.group)
            out.append(t.cpu().numpy())
        return out[0], out[1], out[2], tt


def lockstep(solvers, step=1, check=True):
    """One physical step of all ranks' contexts, driven from this process: the
    requests are fulfilled by copying between the contexts' buffers (the SUM
    in rank order).  Returns the ranks' stats."""
    import torch
    reqs = [abi.DReq() for _ in solvers]
    stats = [abi.Stats() for _ in solvers]
    device = solvers[0]._device
    while True:
        codes = [s.lib.dstep(s.ctx, step, C.byref(r), C.byref(st)) for s, r, st in zip(solvers, reqs, stats)]
        kinds = {r.kind for r in reqs}
        if len(kinds) != 1:
            raise RuntimeError("ranks issued different requests: %s" % sorted(kinds))
        kind = reqs[0].kind
        if kind == abi.DREQ_DONE:
            break
        if device:
            torch.cuda.synchronize()
        if kind == abi.DREQ_REDUCE:
            ns, nm = reqs[0].nsum, reqs[0].nmin
            views = [s.buffer(r.buf, ns + nm) for s, r in zip(solvers, reqs)]
            tot = views[0][:ns].clone()
            for v in views[1:]:
                tot += v[:ns]
            low = views[0][ns:].clone()
            for v in views[1:]:
                low = torch.minimum(low, v[ns:])
            for v in views:
                v[:ns] = tot
                v[ns:] = low
        else:
            seg = reqs[0].seg
            views = [s.buffer(r.buf, seg * r.nranks) for s, r in zip(solvers, reqs)]
            for q, src in enumerate(views):
                for k, dst in enumerate(views):
                    if k != q:
                        dst[q * seg:(q + 1) * seg] = src[q * seg:(q + 1) * seg]
        if device:
            torch.cuda.synchronize()
    if check:
        for s, code in zip(solvers, codes):
            s._check(code, "dstep")
    return stats
