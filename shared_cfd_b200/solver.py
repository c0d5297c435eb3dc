"""Host-side driver of the C ABI: the Python counterpart of the generated
Fortran main program (store/core/main.{head,body.raw,foot}.f90).

A `Case` holds everything the reference reads at start-up (grid, connectivity,
boundary set-up, control parameters, chemistry tables, initial state) in the
reference's own array layout; `Solver` runs it through a library that exports
the ABI of include/scfd_b200.h.
"""
import ctypes as C
import os

import numpy as np

from . import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libscfd_b200.so")


class CudaLibraryMissing(RuntimeError):
    pass


_LIB = None


def load_library(path=None):
    """The CUDA library.  There is no fallback: a missing library is an error."""
    global _LIB
    if path is None and _LIB is not None:
        return _LIB
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise CudaLibraryMissing("%s not built; run `python -m shared_cfd_b200.build`" % p)
    b = abi.Bound(C.CDLL(p), "scfd_")
    if b.abi_version() != abi.ABI_VERSION:
        raise RuntimeError("ABI version mismatch")
    if path is None:
        _LIB = b
    return b


class SolverError(RuntimeError):
    def __init__(self, code, msg=""):
        self.code = code
        super().__init__("%s (%d) %s" % (abi.STATUS_NAMES.get(code, "?"), code, msg))


class Case:
    """All inputs of one run, in the reference's conventions.

    planes: list of (xh, rh) node arrays of shape (ni+1, nj+1)
    desc:   abi.Desc (sizes are filled in from planes)
    cut:    list of 11-int connectivity records
    bcs:    list of abi.BC
    chem:   abi.Chem or None
    q, w, vhi: reference-layout arrays of shape (nplane, njmax+4, nimax+4, K)
    """

    def __init__(self, planes, desc, cut=(), bcs=(), chem=None):
        self.planes = planes
        self.desc = desc
        self.cut = [list(r) for r in cut]
        self.bcs = list(bcs)
        self.chem = chem
        self.desc.abi_version = abi.ABI_VERSION
        self.desc.nplane = len(planes)
        for p, (xh, _) in enumerate(planes):
            self.desc.ni[p] = xh.shape[0] - 1
            self.desc.nj[p] = xh.shape[1] - 1
        self.ni = [xh.shape[0] - 1 for xh, _ in planes]
        self.nj = [xh.shape[1] - 1 for xh, _ in planes]
        self.nimax, self.njmax = max(self.ni), max(self.nj)
        self.nY = desc.ny
        self.D = self.nY + 3
        self.W = self.D + 5
        shape = (len(planes), self.njmax + 4, self.nimax + 4)
        self.q = np.zeros(shape + (self.D,))
        self.w = np.zeros(shape + (self.W,))
        self.vhi = np.zeros(shape + (self.nY,))

    @property
    def ncells(self):
        return sum(a * b for a, b in zip(self.ni, self.nj))

    def interior(self, arr, p):
        """View of plane p's interior cells of a reference-layout array,
        indexed [j-1, i-1, k]."""
        return arr[p, 2:self.nj[p] + 2, 2:self.ni[p] + 2]


class Solver:
    """Runs a Case through one library (the CUDA library by default)."""

    def __init__(self, case, lib=None, partition=None):
        """partition: optional (owner, nranks, rank) of a block-sharded run,
        owner[p] the 0-based rank of plane p (scfd_set_partition)."""
        self.case = case
        self.lib = lib if lib is not None else load_library()
        self.ctx = C.c_void_p()
        self._check(self.lib.create(C.byref(case.desc), C.byref(self.ctx)), "create")
        try:
            if partition is not None:
                owner, nranks, rank = partition
                own = np.ascontiguousarray(owner, dtype=np.int32)
                self._check(self.lib.set_partition(self.ctx, own.ctypes.data_as(C.POINTER(C.c_int32)), nranks,
                                                   rank), "set_partition")
            for p, (xh, rh) in enumerate(case.planes):
                xf = np.asfortranarray(xh, dtype=np.float64).reshape(-1, order="F").copy()
                rf = np.asfortranarray(rh, dtype=np.float64).reshape(-1, order="F").copy()
                self._check(self.lib.set_geometry(self.ctx, p + 1, abi.dptr(xf), abi.dptr(rf)), "set_geometry")
            if case.cut:
                recs = np.ascontiguousarray(np.array(case.cut, dtype=np.int32).reshape(-1))
                self._check(self.lib.set_connectivity(self.ctx, recs.ctypes.data_as(C.POINTER(C.c_int32)),
                                                      len(case.cut)), "set_connectivity")
            if case.bcs:
                arr = (abi.BC * len(case.bcs))(*case.bcs)
                self._check(self.lib.set_bc(self.ctx, arr, len(case.bcs)), "set_bc")
            if case.chem is not None:
                self._check(self.lib.set_chem(self.ctx, C.byref(case.chem)), "set_chem")
            self._check(self.lib.commit(self.ctx), "commit")
        except Exception:
            self.close()
            raise

    def _check(self, code, what=""):
        if code != 0:
            buf = C.create_string_buffer(512)
            if self.ctx:
                self.lib.last_error(self.ctx, buf, 512)
            raise SolverError(code, "%s: %s" % (what, buf.value.decode(errors="replace")))

    def close(self):
        if self.ctx:
            self.lib.destroy(self.ctx)
            self.ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, q=None, w=None, vhi=None, tt=0.0):
        c = self.case
        q = np.ascontiguousarray(c.q if q is None else q, dtype=np.float64)
        w = np.ascontiguousarray(c.w if w is None else w, dtype=np.float64)
        vhi = np.ascontiguousarray(c.vhi if vhi is None else vhi, dtype=np.float64)
        self._check(self.lib.upload(self.ctx, abi.dptr(q), abi.dptr(w), abi.dptr(vhi), tt), "upload")

    def prepare(self, step=1):
        self._check(self.lib.prepare(self.ctx, step), "prepare")

    def step(self, step=1, check=True):
        st = abi.Stats()
        code = self.lib.step(self.ctx, step, C.byref(st))
        if check:
            self._check(code, "step")
        return st

    def run(self, step, nsteps, check=True):
        st = abi.Stats()
        code = self.lib.run(self.ctx, step, nsteps, C.byref(st))
        if check:
            self._check(code, "run")
        return st

    def rms(self):
        r = C.c_double()
        self._check(self.lib.rms(self.ctx, C.byref(r)), "rms")
        return r.value

    def inner_log(self):
        """(omega, res) per inner iteration of the last step, as arrays: omega
        from the Dqrate limiter before the omega_max cap (1e300 when no species
        decreases), res the residual sum (res / res[0] is the reference's
        internal_res.dat ratio)."""
        n = abi.INNER_LOG
        om = np.zeros(n)
        res = np.zeros(n)
        m = self.lib.inner_log(self.ctx, abi.dptr(om), abi.dptr(res), n)
        if m < 0:
            self._check(-m, "inner_log")
        return om[:m], res[:m]

    def download(self):
        c = self.case
        q = np.zeros_like(c.q)
        w = np.zeros_like(c.w)
        vhi = np.zeros_like(c.vhi)
        tt = C.c_double()
        self._check(self.lib.download(self.ctx, abi.dptr(q), abi.dptr(w), abi.dptr(vhi), C.byref(tt)), "download")
        return q, w, vhi, tt.value

    def download_qp(self):
        qp = np.zeros_like(self.case.q)
        self._check(self.lib.download_qp(self.ctx, abi.dptr(qp)), "download_qp")
        return qp

    def write_restart(self, path, step):
        """restart.bin / result file of out_bin (store/core/inout.f90:1-75)."""
        self._check(self.lib.write_restart(self.ctx, os.fsencode(path), step), "write_restart")

    def read_restart(self, path):
        """restart_bin (inout.f90:77-100); returns (step, tt)."""
        step, tt = C.c_int(), C.c_double()
        self._check(self.lib.read_restart(self.ctx, os.fsencode(path), C.byref(step), C.byref(tt)), "read_restart")
        return step.value, tt.value

    def write_geometry(self, path):
        """geometry.bin of out_geo_bin (store/dim/2d/geometry.f90:182-193)."""
        self._check(self.lib.write_geometry(self.ctx, os.fsencode(path)), "write_geometry")

    def tuning(self):
        """The autotuner's choices and candidate times for this context (dict)."""
        import json
        buf = C.create_string_buffer(4096)
        self._check(self.lib.tuning(self.ctx, buf, 4096), "tuning")
        return json.loads(buf.value.decode())

    def stream(self):
        s = C.c_void_p()
        self._check(self.lib.get_stream(self.ctx, C.byref(s)), "get_stream")
        return s.value

    def launch_count(self):
        n = C.c_int64()
        self._check(self.lib.launch_count(self.ctx, C.byref(n)), "launch_count")
        return n.value
