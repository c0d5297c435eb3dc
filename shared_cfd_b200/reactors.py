"""Batched constant-volume 0-D reactors through the C ABI (scfd_reactors_*).

    from shared_cfd_b200 import cases
    from shared_cfd_b200.reactors import Reactors
    m, chem, T0, vrho0, _ = cases.reactor_batch(8192)
    with Reactors(chem, len(T0)) as r:
        out = r.run(T0, vrho0, t_end=2e-3)      # dict of numpy arrays

Each reactor is advanced by reaction_chemeq2 calls
(store/therm_lib/chemkin/core/sub_chem.f90:1684-1713) over dt_call up to
t_end, with the ignition delay of reaction_one_steps (sub_chem.f90:1467-1472).
`lib` selects another library exposing the same entry points (the CPU
restatement, prefix orc_); the default loads the CUDA library and fails if it
is missing.
"""
import ctypes as C

import numpy as np

from . import abi
from .solver import load_library


class Reactors:
    def __init__(self, chem, n_max, lib=None):
        self.lib = lib if lib is not None else load_library()
        self.chem = chem
        self.ns = chem.ns
        self.n_max = int(n_max)
        self.h = C.c_void_p()
        code = self.lib.reactors_create(C.byref(chem), self.n_max, C.byref(self.h))
        if code:
            raise RuntimeError("reactors_create failed: %d" % code)

    def close(self):
        if self.h:
            self.lib.reactors_destroy(self.h)
            self.h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def desc(self, n, t_end, mode=abi.REACTOR_QUEUE, dT_ign=400.0, max_substeps=0, dt_call=1e-6):
        d = abi.ReactorDesc()
        d.abi_version = abi.ABI_VERSION
        d.n, d.mode, d.max_substeps = int(n), int(mode), int(max_substeps)
        d.t_end, d.dT_ign, d.dt_call = float(t_end), float(dT_ign), float(dt_call)
        return d

    def upload(self, T0, vrho0):
        T0 = np.ascontiguousarray(T0, dtype=np.float64)
        vrho0 = np.ascontiguousarray(vrho0, dtype=np.float64).reshape(len(T0), self.ns)
        code = self.lib.reactors_upload(self.h, len(T0), abi.dptr(T0), abi.dptr(vrho0))
        if code:
            raise RuntimeError("reactors_upload failed: %d" % code)
        return len(T0)

    def launch(self, d):
        code = self.lib.reactors_launch(self.h, C.byref(d))
        if code:
            raise RuntimeError("reactors_launch failed: %d" % code)

    def download(self, n):
        out = {"T_end": np.zeros(n), "vrho_end": np.zeros((n, self.ns)), "t_ign": np.zeros(n),
               "evals": np.zeros(n, dtype=np.int64), "flags": np.zeros(n, dtype=np.int32)}
        out["status"] = self.lib.reactors_download(
            self.h, abi.dptr(out["T_end"]), abi.dptr(out["vrho_end"]), abi.dptr(out["t_ign"]),
            out["evals"].ctypes.data_as(C.POINTER(C.c_int64)), out["flags"].ctypes.data_as(C.POINTER(C.c_int32)))
        return out

    def run(self, T0, vrho0, t_end, mode=abi.REACTOR_QUEUE, dT_ign=400.0, max_substeps=0, dt_call=1e-6):
        n = self.upload(T0, vrho0)
        self.launch(self.desc(n, t_end, mode, dT_ign, max_substeps, dt_call))
        return self.download(n)

    def stream(self):
        return self.lib.reactors_stream(self.h)

    def launch_count(self):
        n = C.c_int64()
        self.lib.reactors_launch_count(self.h, C.byref(n))
        return n.value
