"""scfd_rms_noalloc: the convergence RMS for callers that cannot allocate device
memory (their device arrays come from their own data regions or pool, and the
libraries they link may not call cudaMalloc).  It is checked through the C ABI
against scfd_rms, the entry point that uses the context's own scratch, on two
calls in a row with different data.  This file is collected last on purpose:
a failure here leaves every other test already run."""
import ctypes as C

import numpy as np
import pytest

from shared_cfd_b200 import abi, cases
from shared_cfd_b200.solver import Solver

pytestmark = pytest.mark.gpu


def _bind(lib):
    f = lib.lib.scfd_rms_noalloc
    f.restype = C.c_int
    f.argtypes = [C.POINTER(abi.Desc), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    return f


def test_rms_noalloc_matches_context_rms_twice(gpu):
    import torch
    f = _bind(gpu)
    case = cases.perturb(cases.forward_step(2, n=12), seed=4)   # two planes of different shapes
    s = Solver(case, lib=gpu)
    try:
        s.upload()
        s.prepare(1)
        out = torch.zeros(1, dtype=torch.float64, device="cuda")
        for call in range(2):
            s.run(1 + 3 * call, 3)
            want = s.rms()
            q, _, _, _ = s.download()
            qp = s.download_qp()
            dq = torch.from_numpy(np.ascontiguousarray(q)).cuda()
            dqp = torch.from_numpy(np.ascontiguousarray(qp)).cuda()
            torch.cuda.synchronize()
            code = f(C.byref(case.desc), C.c_void_p(dq.data_ptr()), C.c_void_p(dqp.data_ptr()),
                     C.c_void_p(out.data_ptr()), None)
            assert code == abi.OK
            torch.cuda.synchronize()
            got = float(out.item())
            assert want > 0.0
            assert abs(got - want) <= 1e-10 * want, (call, got, want)
    finally:
        s.close()


def test_rms_noalloc_rejects_more_planes_than_its_scratch(gpu):
    f = _bind(gpu)
    d = abi.Desc()
    d.abi_version = abi.ABI_VERSION
    d.ny = 1
    one = C.c_double()
    # 0x04000001 * 64 wraps to 64 in 32-bit arithmetic: the check must not multiply
    for n in (abi.MAX_PLANES + 1, 0x04000001, -1, 0):
        d.nplane = n
        assert f(C.byref(d), C.c_void_p(1), C.c_void_p(1), C.byref(one), None) == abi.E_ARG
