"""scfd_upload / scfd_download with page-locked host arrays (moved by DMA
without the library's staging chunks) against the same calls with pageable
arrays: the same state reaches the device, the same steps run, and the same
bytes come back."""
import ctypes as C

import numpy as np
import pytest

from shared_cfd_b200 import abi, cases
from shared_cfd_b200.solver import Solver

pytestmark = pytest.mark.gpu


def _run(gpu, case, pin):
    import torch

    def host(a):
        a = np.ascontiguousarray(a)
        if not pin:
            return None, a.copy()
        t = torch.empty(a.shape, dtype=torch.float64).pin_memory()
        h = t.numpy()
        h[...] = a
        return t, h

    keep = [host(a) for a in (case.q, case.w, case.vhi, np.zeros_like(case.q))]
    q, w, vhi, qout = (h for _, h in keep)
    s = Solver(case, lib=gpu)
    try:
        lib = s.lib
        s._check(lib.upload(s.ctx, abi.dptr(q), abi.dptr(w), abi.dptr(vhi), 0.0), "upload")
        for k in range(2):
            st = abi.Stats()
            assert lib.step(s.ctx, k + 1, C.byref(st)) == 0
        ttc = C.c_double()
        s._check(lib.download(s.ctx, abi.dptr(qout), None, None, C.byref(ttc)), "download")
        return qout.copy(), ttc.value
    finally:
        s.close()


@pytest.mark.parametrize("make", [lambda: cases.reacting_step(scale=0.0625, inner=2),
                                  lambda: cases.flat_plate(48, 40)])
def test_pinned_and_pageable_copies_agree(gpu, make):
    case = make()
    a, ta = _run(gpu, case, pin=False)
    b, tb = _run(gpu, case, pin=True)
    assert ta == tb
    assert np.array_equal(a, b)
    assert np.isfinite(a).all()
